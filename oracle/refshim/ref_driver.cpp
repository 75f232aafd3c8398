/*
 * ref_driver.cpp -- drives the reference's own host code (g_ACO, OpenclEnv,
 * Problem, read_instance_file) on the fake OpenCL runtime.  TEST INFRASTRUCTURE
 * ONLY; built into oracle/_ref/libcvrp_ref.so by oracle/build_ref.sh.
 *
 * It follows main.cpp:61-94 for one try: read the instance, init_problem, build
 * OpenclEnv + g_ACO, init_aco, then run_aco_iteration + iteration++.  With
 * ls_flag set, g_ACO::local_search is called right after construct_solutions,
 * where the reference has it commented out (g_aco.cpp:84-86 and :127-129);
 * with ls_flag clear, the reference's own init_aco / run_aco_iteration run.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>

#include "io.h"
#include "problem.h"
#include "timer.h"
#include "utilities.h"
#include "vrpHelper.h"
#define private public
#include "gpu/g_aco.h"
#include "gpu/g_type.h"
#include "localSearch.h"
#include "neighbourSearch.h"
#undef private

extern "C" {
extern int fcl_max_wg;
extern long fcl_fake_time;
void *fcl_mem_data(cl_mem m);
size_t fcl_mem_size(cl_mem m);
}

namespace {
struct Session {
    Problem *inst = nullptr;
    OpenclEnv *env = nullptr;
    g_ACO *aco = nullptr;
    int ls_flag = 0;
};
Session *g_s = nullptr;
} // namespace

extern "C" {

/* workdir must contain gpu/kernel.cl (any content): g_type.cpp:21,177-186 reads
 * it relative to the current directory before building the program. */
int ref_open(const char *vrp_path, const char *workdir, int n_ants, int nloc, int seed_time,
             int rnd_seed0, int nn_ls, int ls_flag)
{
    if (g_s) return -1;
    fcl_fake_time = seed_time;
    fcl_max_wg = 4 * nloc; /* cs_grp_size = maxWorkGroupSize / 4, g_aco.cpp:41 */
    g_s = new Session;
    Problem *inst = new Problem(0);
    start_timers();
    read_instance_file(inst, vrp_path);
    init_problem(inst);
    if (n_ants > 0) inst->n_ants = n_ants;
    inst->rnd_seed = rnd_seed0;
    if (nn_ls > 0) inst->nn_ls = nn_ls; /* prefix of the depth max(nn_ls, nn_ants) lists */
    inst->ls_flag = ls_flag != 0;
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return -2;
    if (chdir(workdir) != 0) return -3;
    g_s->env = new OpenclEnv(*inst);
    if (chdir(cwd) != 0) return -4;
    g_s->aco = new g_ACO(*g_s->env, *inst);
    g_s->inst = inst;
    g_s->ls_flag = ls_flag;
    return 0;
}

int ref_init_aco(void)
{
    if (!g_s) return -1;
    g_ACO &a = *g_s->aco;
    Problem &instance = *g_s->inst;
    if (!g_s->ls_flag) {
        a.init_aco();
        return 0;
    }
    /* g_ACO::init_aco (g_aco.cpp:63-93) with the local search enabled */
    instance.best_so_far_time = elapsed_time(REAL);
    instance.iteration = 0;
    instance.best_so_far_ant->tour_length = INFINITY;
    instance.iter_stagnate_cnt = 0;
    instance.best_stagnate_cnt = 0;
    a.create_memory_objects();
    float trail_0 = 0.5;
    a.pheromone_init(trail_0);
    a.construct_solutions();
    a.local_search();
    a.update_statistics();
    a.update_best_so_far_from_device();
    trail_0 = 1.0f / ((rho)*instance.best_so_far_ant->tour_length);
    a.pheromone_init(trail_0);
    instance.iteration++;
    return 0;
}

int ref_run_iteration(void)
{
    if (!g_s) return -1;
    g_ACO &a = *g_s->aco;
    if (!g_s->ls_flag) {
        a.run_aco_iteration();
    } else { /* g_aco.cpp:122-134 with :127-129 enabled */
        a.construct_solutions();
        a.local_search();
        a.update_statistics();
        a.pheromone_update();
    }
    g_s->inst->iteration++; /* main.cpp:86 */
    return 0;
}

/* copy a device buffer out: 0 seeds, 1 solutions, 2 lens, 3 pheromone,
 * 4 total_info, 5 elite ids, 6 bsf records, 7 num_bsf, 8 distance, 9 nn_list,
 * 10 update flag.  Returns the buffer size in bytes (copies min(size, cap)). */
long ref_read(int which, void *dst, long cap)
{
    if (!g_s) return -1;
    g_ACO &a = *g_s->aco;
    cl_mem m = nullptr;
    switch (which) {
    case 0: m = a.seed_mem; break;
    case 1: m = a.solutions_mem; break;
    case 2: m = a.solution_lens_mem; break;
    case 3: m = a.pheromone_mem; break;
    case 4: m = a.total_info_mem; break;
    case 5: m = a.elite_ids_mem; break;
    case 6: m = a.bsf_records_mem; break;
    case 7: m = a.num_bsf_mem; break;
    case 8: m = a.distance_mem; break;
    case 9: m = a.nn_list_mem; break;
    case 10: m = a.update_flag_mem; break;
    default: return -2;
    }
    long size = (long)fcl_mem_size(m);
    if (dst && cap > 0) memcpy(dst, fcl_mem_data(m), (size_t)(cap < size ? cap : size));
    return size;
}

/* host-side Problem fields after init_problem: n, n_ants, nn_ls, capacity,
 * and the host distance matrix / NN lists (compute_distances, compute_nn_lists) */
int ref_problem_info(int *out4)
{
    if (!g_s) return -1;
    out4[0] = g_s->inst->num_node;
    out4[1] = g_s->inst->n_ants;
    out4[2] = g_s->inst->nn_ls;
    out4[3] = g_s->inst->vehicle_capacity;
    return 0;
}

int ref_host_check_solution(const int *tour, int tour_size)
{
    if (!g_s) return -1;
    return check_solution(g_s->inst, const_cast<int *>(tour), tour_size) ? 1 : 0;
}

void ref_close(void)
{
    if (!g_s) return;
    delete g_s->aco;
    delete g_s->env;
    g_s = nullptr; /* Problem and its matrices are leaked on purpose: exit_problem
                      frees a new-allocated object with free() (problem.cpp:76) */
}

/* read_instance_file + init_problem only: the reader, distance matrix and NN
 * lists of the reference host code for an instance file. */
int ref_read_instance(const char *vrp_path, int *n_out, int *capacity_out, float *x, float *y, int *demand,
                      float *dist, int *nn, int cap_nodes, int *nn_depth_out, float *optimum_out,
                      float *max_dist_out, float *serv_time_out)
{
    Problem *inst = new Problem(0);
    read_instance_file(inst, vrp_path);
    init_problem(inst);
    int n = inst->num_node;
    *n_out = n;
    *capacity_out = inst->vehicle_capacity;
    if (optimum_out) *optimum_out = inst->optimum;
    if (max_dist_out) *max_dist_out = inst->max_distance;
    if (serv_time_out) *serv_time_out = inst->service_time;
    int depth = inst->nn_ls > inst->nn_ants ? inst->nn_ls : inst->nn_ants;
    if (depth >= n) depth = n - 1;
    *nn_depth_out = depth;
    if (n <= cap_nodes) {
        for (int i = 0; i < n; i++) {
            x[i] = inst->nodeptr[i].x;
            y[i] = inst->nodeptr[i].y;
            demand[i] = inst->nodeptr[i].demand;
            for (int j = 0; j < n; j++) dist[(size_t)i * n + j] = inst->distance[i][j];
            for (int j = 0; j < depth; j++) nn[(size_t)i * depth + j] = inst->nn_list[i][j];
        }
    }
    return 0;
}

/* The reference's CPU inter-route swap (LocalSearch::swap, localSearch.cpp:301-410)
 * applied in place to one tour of the instance in vrp_path (read_instance_file +
 * init_problem; no OpenCL state involved). */
int ref_swap(const char *vrp_path, int *tour, int tour_size)
{
    Problem *inst = new Problem(0);
    read_instance_file(inst, vrp_path);
    init_problem(inst);
    LocalSearch ls(inst);
    ls.swap(tour, tour_size);
    return 0; /* inst leaked on purpose, as in ref_read_instance */
}

/* `count` proposals of the reference's NeighbourSearch::search
 * (neighbourSearch.cpp:72-95) on one tour of the instance in vrp_path, with
 * libc's generator seeded by srandom(seed); with `apply`, the valid proposals
 * whose gain is below -EPSILON are applied (Move::apply, move.cpp) before the
 * next one.  type -1 marks a proposal the reference returns as NULL. */
int ref_ns(const char *vrp_path, int *tour, int tour_size, unsigned seed, int count, int apply, int *type,
           int *valid, float *gain, int *pos1, int *pos2)
{
    Problem *inst = new Problem(0);
    read_instance_file(inst, vrp_path);
    init_problem(inst);
    NeighbourSearch ns(inst);
    srandom(seed);
    AntStruct ant;
    ant.tour = tour;
    ant.tour_size = tour_size;
    ant.tour_length = 0;
    for (int k = 0; k < count; k++) {
        Move *m = ns.search(&ant);
        if (!m) {
            type[k] = -1; valid[k] = 0; gain[k] = 0; pos1[k] = pos2[k] = 0;
            continue;
        }
        type[k] = (int)m->type; valid[k] = m->valid; gain[k] = m->gain; pos1[k] = m->pos_n1; pos2[k] = m->pos_n2;
        if (apply && m->valid && m->gain < -EPSILON) m->apply();
        delete m;
    }
    return 0;
}

} /* extern "C" */
