// host.h -- host-side pieces of the path that stay on the CPU: the VRPLIB
// reader, distances, NN lists, seeds, validation, and the small lookup tables
// the kernels need (tie priorities of the I-Roulette tournament, RNG jump
// multipliers).  Each function names the reference routine it replaces.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace aco {

constexpr float kEpsilon = 0.001f;         // utilities.h:19, kernel.cl:6
constexpr uint32_t kIM = 2147483647u;      // Park-Miller modulus (utilities.h:37)
constexpr uint32_t kIA = 16807u;           // multiplier (utilities.h:36)

struct VrpFile {
    std::string name;
    int n = 0;
    std::vector<float> x, y;
    std::vector<int> demand;
    int capacity = 0;
    float max_distance = 0, service_time = 0, optimum = 0;
    int dist_type = 0;
};

// read_instance_file (io.cpp:334-517).  Returns 0 or ACO_ERR_IO.
int read_vrplib(const char *path, VrpFile &out, std::string &err);

// compute_distances (vrpHelper.cpp:160-184).
void compute_distances(int n, const float *x, const float *y, int dist_type, float *dist);
// One entry of that matrix.
float point_distance(const float *x, const float *y, int dist_type, int i, int j);

// compute_nn_lists (vrpHelper.cpp:188-236); returns the depth actually used.
int compute_nn_lists(int n, const float *dist, int nn_ls, int nn_ants, std::vector<int> &nn);

// check_solution / check_route (problem.cpp:226-319).
bool check_solution(int n, const float *dist, const int *demand, int capacity, float max_dist,
                    float serv_time, const int *tour, int tour_size);

// compute_tour_length (vrpHelper.cpp:244-253) and its fp64 twin.
float tour_length32(int n, const float *dist, const int *tour, int tour_size);
double tour_length64(int n, const float *dist, const int *tour, int tour_size);

// ran01 (utilities.cpp:271-288).
float ran01(int *idum);
// seed generation (g_aco.cpp:714-722) with time(NULL) = seed_time.
void make_seeds(int seed_time, int *rnd_seed, int n_ants, int nloc, int *seeds);

// Rank at which each node wins ties in the I-Roulette tournament
// (kernel.cl:340-366): prio[node], 0 = preferred.
std::vector<int> tournament_priority(int n);

// 16807^e mod (2^31-1).
uint32_t pm_pow(uint64_t e);
// x mod (2^31-1) in [0, 2^31-1): the state one Schrage step acts on.
uint32_t pm_normalize(int x);

} // namespace aco
