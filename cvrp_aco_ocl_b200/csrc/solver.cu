// solver.cu -- the C ABI of include/cvrp_aco.h: g_ACO's lifecycle
// (cvrp_ocl/gpu/g_aco.cpp) on one CUDA stream of one B200.
//
// aco_create   = g_ACO::g_ACO + create_memory_objects (g_aco.cpp:35-43, 640-761)
// aco_init     = g_ACO::init_aco (g_aco.cpp:63-93)
// aco_iterate  = run_aco_iteration (g_aco.cpp:122-134) + iteration++ (main.cpp:86),
//                replayed as one CUDA graph of four kernels:
//                construct -> 2-opt -> stats (best, bsf, elites, deposit list)
//                -> fused evaporation/deposit/total_info pass.
// All state stays on the device; the host synchronises once per aco_iterate
// call and reads a 4-byte status word.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cvrp_aco.h"
#include "host.h"
#include "kernels.h"

using namespace aco;

struct aco_solver {
    aco_params p{};
    int n = 0, A = 0, T = 0, ld = 0, n4 = 0, nloc = 0, lg = 0, kmax = 0, nn_ls = 0, K = 0, Kp = 0, R = 0;
    int capacity = 0;
    float max_dist = 0, serv_time = 0;
    int alpha_int = -1, beta_int = -1;
    int dev = 0, sm_count = 148;
    cudaStream_t st = nullptr;
    std::vector<float> dist_h;
    std::vector<int> demand_h;
    std::vector<void *> allocs;
    float *d_dist = nullptr, *d_heur = nullptr, *d_tau = nullptr, *d_total = nullptr;
    int *d_demand = nullptr, *d_nnls = nullptr, *d_seeds = nullptr, *d_sol = nullptr;
    uint32_t *d_key = nullptr, *d_jump = nullptr, *d_adv = nullptr, *d_depmask = nullptr;
    uint16_t *d_nn16 = nullptr;
    uint32_t *d_cand32 = nullptr;
    float *d_lens = nullptr, *d_dtau = nullptr;
    int *d_elites = nullptr, *d_succ = nullptr, *d_num_bsf = nullptr, *d_iter = nullptr, *d_status = nullptr;
    aco_record *d_records = nullptr;
    unsigned long long *d_t0 = nullptr;
    int *h_pin = nullptr; // [0] status, [1] iteration, [2..3] bsf length bits
    int cp_wpa = 1, cp_apc = 1, cn_apc = 1, ls_apc = 1, ls_rmax = 64;
    bool cp_stage = false, cn_stage = false, cn_packed = false, ls_snn = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool initialized = false;
    std::chrono::steady_clock::time_point t_init;
};

namespace {

#define CK(x)                                                                                                  \
    do {                                                                                                       \
        cudaError_t e_ = (x);                                                                                  \
        if (e_ != cudaSuccess) return ACO_ERR_CUDA;                                                            \
    } while (0)

constexpr size_t kSmemBudget = 227 * 1024;

int exp_as_int(float e)
{
    if (e >= 0.0f && e <= 8.0f && e == (float)(int)e) return (int)e;
    return -1;
}

template <class T> int dalloc(aco_solver *s, T **ptr, size_t count)
{
    void *p = nullptr;
    if (cudaMalloc(&p, count * sizeof(T) + 16) != cudaSuccess) return ACO_ERR_NOMEM;
    if (cudaMemset(p, 0, count * sizeof(T) + 16) != cudaSuccess) return ACO_ERR_CUDA;
    s->allocs.push_back(p);
    *ptr = static_cast<T *>(p);
    return ACO_OK;
}

int ilog2(int v)
{
    int r = 0;
    while ((1 << r) < v) r++;
    return r;
}

void free_all(aco_solver *s)
{
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->exec = nullptr;
    s->graph = nullptr;
    for (void *p : s->allocs) cudaFree(p);
    s->allocs.clear();
    if (s->h_pin) cudaFreeHost(s->h_pin);
    s->h_pin = nullptr;
    if (s->st) cudaStreamDestroy(s->st);
    s->st = nullptr;
}

// Launch configuration: ants per CTA so that the grid covers the SMs, warps
// per ant so that every thread owns at most 32 nodes of a row, and shared-memory
// staging wherever the 227 KB budget allows.
void pick_config(aco_solver *s)
{
    const int A = s->A, n = s->n;
    auto per_block = [&](int sms) { return std::max(1, std::min(8, (A + sms - 1) / sms)); };
    int wpa = 1;
    while (wpa < 8 && 32 * wpa * 32 < n) wpa *= 2;
    while (wpa < 8 && n > 256 * wpa && 32 * wpa * 2 <= s->nloc) wpa *= 2;
    wpa = std::min(wpa, s->nloc / 32);
    if (s->p.warps_per_ant > 0) wpa = s->p.warps_per_ant;
    s->cp_wpa = wpa;
    s->cp_apc = s->p.ants_per_block > 0 ? s->p.ants_per_block : std::max(1, per_block(s->sm_count) / wpa);
    const bool fin = !std::isinf(s->max_dist);
    s->cp_stage = construct_parity_smem(n, s->nloc, s->kmax, wpa, s->cp_apc, true, fin) <= kSmemBudget;
    s->cn_apc = s->p.ants_per_block > 0 ? s->p.ants_per_block : per_block(s->sm_count);
    // throughput construct: pack (node | demand << 16) when demands fit 16 bits,
    // stage the full matrix when it fits next to the candidate tables
    int maxdem = 0, mindem = 0;
    for (int i = 0; i < n; i++) {
        maxdem = std::max(maxdem, s->demand_h[i]);
        mindem = std::min(mindem, s->demand_h[i]);
    }
    const bool packable = maxdem <= 0xFFFF && mindem >= 0;
    s->cn_packed = false;
    s->cn_stage = false;
    if (s->K > 0) {
        for (int apc = s->cn_apc; apc >= 1 && !s->cn_stage; apc--) {
            if (packable && n <= 1024 && construct_nn_smem(n, s->K, s->Kp, apc, true, true) <= kSmemBudget) {
                s->cn_stage = s->cn_packed = true;
                s->cn_apc = apc;
            }
        }
        if (!s->cn_stage) {
            s->cn_packed = packable && construct_nn_smem(n, s->K, s->Kp, s->cn_apc, false, true) <= kSmemBudget;
            while (s->cn_apc > 1 && construct_nn_smem(n, s->K, s->Kp, s->cn_apc, false, s->cn_packed) > kSmemBudget)
                s->cn_apc--;
        }
    }
    // 2-opt: one CTA per ant, one warp per route (routes estimated from the demand)
    long long dem = 0;
    for (int i = 1; i < n; i++) dem += s->demand_h[i];
    const int est_routes = s->capacity > 0 ? (int)std::min<long long>(n, dem / s->capacity + 1) : 1;
    s->ls_apc = std::max(1, std::min(32, est_routes + 2)); // warps per ant: about one per route
    s->ls_rmax = 32;
    s->ls_snn = false;
    while (s->ls_apc > 1 && local_search_smem(n, s->nn_ls, s->ls_rmax, s->ls_apc, false) > kSmemBudget)
        s->ls_apc--;
}

ConstructArgs cargs(aco_solver *s)
{
    ConstructArgs a{};
    a.n = s->n; a.ld = s->ld; a.n_ants = s->A; a.T = s->T; a.nloc = s->nloc; a.log2_nloc = s->lg; a.kmax = s->kmax;
    a.capacity = s->capacity; a.max_dist = s->max_dist; a.serv_time = s->serv_time;
    a.total = s->d_total; a.dist = s->d_dist; a.demand = s->d_demand; a.tiekey = s->d_key; a.jump = s->d_jump;
    a.adv = s->d_adv; a.nn16 = s->d_nn16; a.cand32 = s->d_cand32; a.K = s->K; a.Kp = s->Kp;
    a.seeds = s->d_seeds; a.solutions = s->d_sol; a.lens = s->d_lens; a.status = s->d_status;
    return a;
}

int do_construct(aco_solver *s)
{
    const ConstructArgs a = cargs(s);
    if (s->p.mode == ACO_MODE_THROUGHPUT) CK(launch_construct_nn(a, s->cn_apc, s->cn_stage, s->cn_packed, s->st));
    else CK(launch_construct_parity(a, s->cp_wpa, s->cp_apc, s->cp_stage, s->st));
    return ACO_OK;
}

int do_local_search(aco_solver *s)
{
    LocalSearchArgs a{};
    a.n = s->n; a.ld = s->ld; a.n_ants = s->A; a.T = s->T; a.nn_ls = s->nn_ls; a.rmax = s->ls_rmax;
    a.pass_limit = s->p.ls_pass_limit;
    a.dist = s->d_dist; a.nn_list = s->d_nnls; a.solutions = s->d_sol; a.lens = s->d_lens; a.status = s->d_status;
    CK(launch_local_search(a, s->ls_apc, s->ls_snn, s->st));
    return ACO_OK;
}

int do_stats(aco_solver *s, bool elites)
{
    StatsArgs a{};
    a.n = s->n; a.n_ants = s->A; a.T = s->T; a.nloc = s->nloc; a.log2_nloc = s->lg; a.ras_ranks = s->R;
    a.record_cap = s->p.record_cap; a.do_elites = elites ? 1 : 0;
    a.solutions = s->d_sol; a.lens = s->d_lens; a.elites = s->d_elites; a.succ = s->d_succ; a.depmask = s->d_depmask;
    a.d_tau = s->d_dtau; a.num_bsf = s->d_num_bsf; a.records = s->d_records; a.iteration = s->d_iter;
    a.t0_ns = s->d_t0; a.status = s->d_status;
    CK(launch_stats(a, s->st));
    return ACO_OK;
}

int do_update(aco_solver *s)
{
    UpdateArgs a{};
    a.n = s->n; a.ld = s->ld; a.q = (s->n + 3) / 4;
    a.qinv = ((1ull << 40) + (unsigned long long)a.q - 1) / (unsigned long long)a.q;
    a.ras_ranks = s->R; a.evap = 1.0f - s->p.rho; a.alpha = s->p.alpha; a.alpha_int = s->alpha_int;
    a.tau = s->d_tau; a.total = s->d_total; a.heur = s->d_heur; a.succ = s->d_succ; a.depmask = s->d_depmask;
    a.d_tau = s->d_dtau;
    CK(launch_pheromone_update(a, s->sm_count, s->st));
    return ACO_OK;
}

int do_pheromone_init(aco_solver *s, float trail, bool from_bsf)
{
    InitArgs a{};
    a.n = s->n; a.ld = s->ld; a.trail = trail; a.from_bsf = from_bsf ? 1 : 0; a.rho = s->p.rho;
    a.alpha = s->p.alpha; a.alpha_int = s->alpha_int; a.bsf_len = s->d_lens + s->A;
    a.tau = s->d_tau; a.total = s->d_total; a.heur = s->d_heur;
    CK(launch_pheromone_init(a, s->st));
    return ACO_OK;
}

int run_iteration_phases(aco_solver *s)
{
    int rc = do_construct(s);
    if (rc == ACO_OK && s->p.ls_flag) rc = do_local_search(s);
    if (rc == ACO_OK) rc = do_stats(s, true);
    if (rc == ACO_OK) rc = do_update(s);
    return rc;
}

int sync_status(aco_solver *s)
{
    CK(cudaMemcpyAsync(s->h_pin, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(s->h_pin + 1, s->d_iter, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return s->h_pin[0];
}

int ensure_graph(aco_solver *s)
{
    if (s->exec) return ACO_OK;
    CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    int rc = run_iteration_phases(s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->st, &g);
    if (rc != ACO_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc != ACO_OK ? rc : ACO_ERR_CUDA;
    }
    s->graph = g;
    CK(cudaGraphInstantiate(&s->exec, g, 0));
    return ACO_OK;
}

int set_device(aco_solver *s)
{
    CK(cudaSetDevice(s->dev));
    return ACO_OK;
}

} // namespace

extern "C" {

int aco_params_default(aco_params *p, int n)
{
    if (!p) return ACO_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->n_ants = n;                 // problem.cpp:189
    p->alpha = 1.0f;               // problem.cpp:207
    p->beta = 2.0f;
    p->rho = 0.1f;
    p->ras_ranks = 6;              // problem.cpp:210
    p->nn_ls = n > 2 ? n - 2 : 0;  // problem.cpp:191-193
    p->nn_ants = std::min(25, n > 2 ? n - 2 : 1);
    p->ls_flag = 1;                // problem.cpp:203
    p->mode = ACO_MODE_PARITY;
    p->nloc = 256;                 // NVIDIA OpenCL maxWorkGroupSize 1024 / 4 (g_aco.cpp:41)
    p->seed_time = 0;
    p->rnd_seed = 0;
    p->max_iteration = 250;        // problem.cpp:196
    p->max_runtime = 600.0f;       // problem.cpp:213
    p->ls_pass_limit = 4096;
    p->record_cap = 4096;          // g_aco.cpp:727-729
    p->device = 0;
    p->use_graph = 1;
    return ACO_OK;
}

int aco_read_vrplib(const char *path, int *n, float *x, float *y, int *demand, int *capacity, float *max_distance,
                    float *service_time, int *dist_type, float *optimum, char *name, int name_cap)
{
    if (!path || !n) return ACO_ERR_INVALID;
    VrpFile f;
    std::string err;
    const int rc = read_vrplib(path, f, err);
    if (rc != ACO_OK) return rc;
    if (x == nullptr) {
        *n = f.n;
        return ACO_OK;
    }
    if (*n < f.n) return ACO_ERR_CAPACITY;
    *n = f.n;
    std::memcpy(x, f.x.data(), sizeof(float) * f.n);
    if (y) std::memcpy(y, f.y.data(), sizeof(float) * f.n);
    if (demand) std::memcpy(demand, f.demand.data(), sizeof(int) * f.n);
    if (capacity) *capacity = f.capacity;
    if (max_distance) *max_distance = f.max_distance;
    if (service_time) *service_time = f.service_time;
    if (dist_type) *dist_type = f.dist_type;
    if (optimum) *optimum = f.optimum;
    if (name && name_cap > 0) {
        std::strncpy(name, f.name.c_str(), (size_t)name_cap - 1);
        name[name_cap - 1] = 0;
    }
    return ACO_OK;
}

int aco_compute_distances(int n, const float *x, const float *y, int dist_type, float *dist)
{
    if (n <= 0 || !x || !y || !dist) return ACO_ERR_INVALID;
    compute_distances(n, x, y, dist_type, dist);
    return ACO_OK;
}

int aco_compute_nn_lists(int n, const float *dist, int nn_ls, int nn_ants, int *nn, int *depth)
{
    if (n <= 1 || !dist || !nn) return ACO_ERR_INVALID;
    std::vector<int> v;
    const int d = compute_nn_lists(n, dist, nn_ls, nn_ants, v);
    std::memcpy(nn, v.data(), sizeof(int) * v.size());
    if (depth) *depth = d;
    return ACO_OK;
}

int aco_check_solution(const aco_instance *inst, const int *tour, int tour_size)
{
    if (!inst || !tour || inst->n <= 0 || !inst->demand) return ACO_ERR_INVALID;
    std::vector<float> d;
    const float *dist = inst->dist;
    if (!dist) {
        if (!inst->x || !inst->y) return ACO_ERR_INVALID;
        d.resize((size_t)inst->n * inst->n);
        compute_distances(inst->n, inst->x, inst->y, inst->dist_type, d.data());
        dist = d.data();
    }
    return check_solution(inst->n, dist, inst->demand, inst->capacity, inst->max_distance, inst->service_time, tour,
                          tour_size)
               ? 1
               : 0;
}

int aco_tour_length(int n, const float *dist, const int *tour, int tour_size, float *len32, double *len64)
{
    if (n <= 0 || !dist || !tour) return ACO_ERR_INVALID;
    for (int i = 0; i < tour_size; i++)
        if (tour[i] < 0 || tour[i] >= n) return ACO_ERR_INVALID;
    if (len32) *len32 = tour_length32(n, dist, tour, tour_size);
    if (len64) *len64 = tour_length64(n, dist, tour, tour_size);
    return ACO_OK;
}

int aco_make_seeds(int seed_time, int *rnd_seed, int n_ants, int nloc, int *seeds)
{
    if (!rnd_seed || !seeds || n_ants <= 0 || nloc <= 0) return ACO_ERR_INVALID;
    make_seeds(seed_time, rnd_seed, n_ants, nloc, seeds);
    return ACO_OK;
}

int aco_create(const aco_instance *inst, const aco_params *params, aco_solver **out)
{
    if (!inst || !out || !inst->demand) return ACO_ERR_INVALID;
    *out = nullptr;
    const int n = inst->n;
    if (n < 2 || n > 32767) return ACO_ERR_INVALID;
    aco_params p;
    if (params) p = *params;
    else aco_params_default(&p, n);
    if (p.n_ants <= 0) p.n_ants = n;
    if (p.nloc < 32 || p.nloc > 1024 || (p.nloc & (p.nloc - 1))) return ACO_ERR_INVALID;
    if (p.ras_ranks < 1 || p.ras_ranks > 32) return ACO_ERR_INVALID;
    if (p.nn_ls < 0 || p.nn_ls > n - 2) return ACO_ERR_INVALID; // depth n-1 would list the node itself
    if (p.mode != ACO_MODE_PARITY && p.mode != ACO_MODE_THROUGHPUT) return ACO_ERR_INVALID;
    if (p.mode == ACO_MODE_THROUGHPUT && (p.nn_ants < 1 || p.nn_ants > 32 || p.nn_ants > n - 1))
        return ACO_ERR_INVALID;
    if (p.warps_per_ant != 0 && (p.warps_per_ant < 1 || p.warps_per_ant > 8 ||
                                 (p.warps_per_ant & (p.warps_per_ant - 1)) || 32 * p.warps_per_ant > p.nloc))
        return ACO_ERR_INVALID;
    if (p.ants_per_block < 0 || p.ants_per_block > 16) return ACO_ERR_INVALID;
    if (p.record_cap <= 0) p.record_cap = 4096;
    if (!(p.rho > 0.0f && p.rho <= 1.0f)) return ACO_ERR_INVALID;

    aco_solver *s = new (std::nothrow) aco_solver;
    if (!s) return ACO_ERR_NOMEM;
    s->p = p;
    s->n = n;
    s->A = p.n_ants;
    s->T = 2 * n;
    s->ld = (n + 31) & ~31;
    s->n4 = (n + 3) & ~3;
    s->nloc = p.nloc;
    s->lg = ilog2(p.nloc);
    s->kmax = (n + p.nloc - 1) / p.nloc;
    s->nn_ls = p.nn_ls;
    s->K = p.mode == ACO_MODE_THROUGHPUT ? p.nn_ants : 0;
    s->Kp = s->K > 0 ? (s->K + 7) & ~7 : 8;
    s->R = p.ras_ranks;
    s->capacity = inst->capacity;
    s->max_dist = inst->max_distance;
    s->serv_time = inst->service_time;
    s->alpha_int = exp_as_int(p.alpha);
    s->beta_int = exp_as_int(p.beta);
    s->dev = p.device;
    if (s->A > 1024 * 1024) {
        delete s;
        return ACO_ERR_INVALID;
    }

    // host inputs: distances (compute_distances) and NN lists (compute_nn_lists)
    s->dist_h.resize((size_t)n * n);
    if (inst->dist) std::memcpy(s->dist_h.data(), inst->dist, sizeof(float) * n * n);
    else {
        if (!inst->x || !inst->y) {
            delete s;
            return ACO_ERR_INVALID;
        }
        compute_distances(n, inst->x, inst->y, inst->dist_type, s->dist_h.data());
    }
    s->demand_h.assign(inst->demand, inst->demand + n);
    for (int i = 1; i < n; i++) { // a customer nobody can serve makes construct loop forever (kernel.cl:438,461)
        if (s->demand_h[i] > s->capacity) {
            delete s;
            return ACO_ERR_INFEASIBLE;
        }
        const float reach = (0.0f + (s->dist_h[i] + s->serv_time)) + s->dist_h[(size_t)i * n];
        if (!(reach <= s->max_dist)) {
            delete s;
            return ACO_ERR_INFEASIBLE;
        }
    }
    std::vector<int> nn;
    const int depth = compute_nn_lists(n, s->dist_h.data(), p.nn_ls, s->K, nn);

    int dc = 0;
    if (cudaGetDeviceCount(&dc) != cudaSuccess || dc <= p.device || p.device < 0) {
        delete s;
        return ACO_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, p.device) != cudaSuccess || prop.major < 10) {
        delete s;
        return ACO_ERR_NO_DEVICE;
    }
    s->sm_count = prop.multiProcessorCount;
    int rc = set_device(s);
    if (rc == ACO_OK && cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) rc = ACO_ERR_CUDA;
    if (rc == ACO_OK && cudaMallocHost(&s->h_pin, 64) != cudaSuccess) rc = ACO_ERR_NOMEM;
    const size_t nl = (size_t)n * s->ld;
    if (rc == ACO_OK) rc = dalloc(s, &s->d_dist, nl);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_heur, nl);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_tau, nl);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_total, nl);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_demand, (size_t)s->n4);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_key, (size_t)s->n4);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_jump, (size_t)((s->kmax + 3) & ~3));
    if (rc == ACO_OK) rc = dalloc(s, &s->d_adv, (size_t)s->nloc);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_nn16, (size_t)n * s->Kp);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_cand32, (size_t)n * s->Kp);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_nnls, (size_t)n * std::max(1, s->nn_ls));
    if (rc == ACO_OK) rc = dalloc(s, &s->d_seeds, (size_t)s->A * s->nloc);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_sol, (size_t)s->T * (s->A + 1) + 1);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_lens, (size_t)s->A + 1);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_elites, (size_t)s->R);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_succ, (size_t)s->R * n);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_depmask, (size_t)n);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_dtau, (size_t)s->R);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_num_bsf, 1);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_records, (size_t)p.record_cap);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_iter, 1);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_status, 1);
    if (rc == ACO_OK) rc = dalloc(s, &s->d_t0, 1);
    if (rc != ACO_OK) {
        free_all(s);
        delete s;
        return rc;
    }

    // lookup tables
    std::vector<int> dem4(s->n4, 0);
    std::copy(s->demand_h.begin(), s->demand_h.end(), dem4.begin());
    const std::vector<int> prio = tournament_priority(n);
    std::vector<uint32_t> key(s->n4, 0);
    for (int i = 0; i < n; i++) key[i] = ((uint32_t)(0xFFFF - prio[i]) << 16) | (uint32_t)i;
    std::vector<uint32_t> jump((s->kmax + 3) & ~3, 0);
    for (int k = 0; k < s->kmax; k++) jump[k] = pm_pow((uint64_t)k + 1);
    std::vector<uint32_t> adv(s->nloc, 1);
    for (int l = 0; l < s->nloc; l++) adv[l] = pm_pow(l < n ? (uint64_t)((n - l + s->nloc - 1) / s->nloc) : 0);
    std::vector<uint16_t> nn16((size_t)n * s->Kp, 0);
    std::vector<uint32_t> cand32((size_t)n * s->Kp, 0); // padding entries: node 0 (always visited)
    for (int i = 0; i < n && s->K > 0; i++)
        for (int j = 0; j < s->K; j++) {
            const int c = nn[(size_t)i * depth + j];
            nn16[(size_t)i * s->Kp + j] = (uint16_t)c;
            cand32[(size_t)i * s->Kp + j] = (uint32_t)c | ((uint32_t)(s->demand_h[c] & 0xFFFF) << 16);
        }
    std::vector<int> nnls((size_t)n * std::max(1, s->nn_ls), 0);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < s->nn_ls; j++) nnls[(size_t)i * s->nn_ls + j] = nn[(size_t)i * depth + j];
    std::vector<int> seeds((size_t)s->A * s->nloc);
    int rs = p.rnd_seed;
    make_seeds(p.seed_time, &rs, s->A, s->nloc, seeds.data());

    cudaStream_t st = s->st;
    auto up = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    };
    bool ok = cudaMemcpy2DAsync(s->d_dist, (size_t)s->ld * 4, s->dist_h.data(), (size_t)n * 4, (size_t)n * 4, n,
                                cudaMemcpyHostToDevice, st) == cudaSuccess;
    ok = ok && up(s->d_demand, dem4.data(), dem4.size() * 4);
    ok = ok && up(s->d_key, key.data(), key.size() * 4);
    ok = ok && up(s->d_jump, jump.data(), jump.size() * 4);
    ok = ok && up(s->d_adv, adv.data(), adv.size() * 4);
    ok = ok && up(s->d_nn16, nn16.data(), nn16.size() * 2);
    ok = ok && up(s->d_cand32, cand32.data(), cand32.size() * 4);
    ok = ok && up(s->d_nnls, nnls.data(), nnls.size() * 4);
    ok = ok && up(s->d_seeds, seeds.data(), seeds.size() * 4);
    ok = ok && launch_heur(s->d_dist, s->d_heur, n, s->ld, p.beta, s->beta_int, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        free_all(s);
        delete s;
        return ACO_ERR_CUDA;
    }
    pick_config(s);
    *out = s;
    return ACO_OK;
}

void aco_destroy(aco_solver *s)
{
    if (!s) return;
    cudaSetDevice(s->dev);
    if (s->st) cudaStreamSynchronize(s->st);
    free_all(s);
    delete s;
}

int aco_init(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    int rc = set_device(s);
    if (rc != ACO_OK) return rc;
    const float inf = INFINITY;
    const int zero = 0;
    CK(cudaMemcpyAsync(s->d_lens + s->A, &inf, sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->d_num_bsf, 0, sizeof(int), s->st));
    CK(cudaMemsetAsync(s->d_iter, 0, sizeof(int), s->st));
    CK(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->st));
    CK(launch_t0(s->d_t0, s->st));
    (void)zero;
    s->t_init = std::chrono::steady_clock::now();
    // g_aco.cpp:79-92
    rc = do_pheromone_init(s, 0.5f, false);
    if (rc == ACO_OK) rc = do_construct(s);
    if (rc == ACO_OK && s->p.ls_flag) rc = do_local_search(s);
    if (rc == ACO_OK) rc = do_stats(s, false);
    if (rc == ACO_OK) rc = do_pheromone_init(s, 0.f, true);
    if (rc != ACO_OK) return rc;
    CK(cudaMemcpyAsync(s->h_pin, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->initialized = s->h_pin[0] == ACO_OK;
    return s->h_pin[0];
}

int aco_iterate(aco_solver *s, int n_iter)
{
    if (!s || n_iter < 0) return ACO_ERR_INVALID;
    if (!s->initialized) return ACO_ERR_STATE;
    int rc = set_device(s);
    if (rc != ACO_OK) return rc;
    if (s->p.use_graph) {
        rc = ensure_graph(s);
        if (rc != ACO_OK) return rc;
        for (int i = 0; i < n_iter; i++) CK(cudaGraphLaunch(s->exec, s->st));
    } else {
        for (int i = 0; i < n_iter && rc == ACO_OK; i++) rc = run_iteration_phases(s);
        if (rc != ACO_OK) return rc;
    }
    return sync_status(s);
}

int aco_run(aco_solver *s, float optimum, int *iterations_done)
{
    if (!s) return ACO_ERR_INVALID;
    int rc = ACO_OK;
    if (!s->initialized) {
        rc = aco_init(s);
        if (rc != ACO_OK) return rc;
    }
    int done = 0;
    for (;;) { // termination_condition (main.cpp:29-34)
        int it = 0;
        float best = 0;
        CK(cudaMemcpyAsync(s->h_pin + 1, s->d_iter, sizeof(int), cudaMemcpyDeviceToHost, s->st));
        CK(cudaMemcpyAsync(s->h_pin + 2, s->d_lens + s->A, sizeof(float), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        it = s->h_pin[1];
        std::memcpy(&best, s->h_pin + 2, sizeof(float));
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t_init).count();
        if (it >= s->p.max_iteration || el >= s->p.max_runtime || std::fabs(best - optimum) < 10 * kEpsilon) break;
        rc = aco_iterate(s, 1);
        if (rc != ACO_OK) break;
        done++;
    }
    if (iterations_done) *iterations_done = done;
    return rc;
}

int aco_construct_solutions(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const int rc = do_construct(s);
    return rc != ACO_OK ? rc : sync_status(s);
}

int aco_local_search(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const int rc = do_local_search(s);
    return rc != ACO_OK ? rc : sync_status(s);
}

int aco_update_statistics(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const int rc = do_stats(s, true);
    return rc != ACO_OK ? rc : sync_status(s);
}

int aco_pheromone_update(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const int rc = do_update(s);
    return rc != ACO_OK ? rc : sync_status(s);
}

int aco_pheromone_init(aco_solver *s, float trail_0)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const int rc = do_pheromone_init(s, trail_0, false);
    return rc != ACO_OK ? rc : sync_status(s);
}

int aco_get_best(aco_solver *s, int *tour, int cap, int *tour_size, float *length)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    std::vector<int> buf(s->T);
    float len = 0;
    CK(cudaMemcpyAsync(buf.data(), s->d_sol + (size_t)s->T * s->A, sizeof(int) * s->T, cudaMemcpyDeviceToHost,
                       s->st));
    CK(cudaMemcpyAsync(&len, s->d_lens + s->A, sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    const int size = buf[s->T - 1];
    if (tour_size) *tour_size = size;
    if (length) *length = len;
    if (tour) {
        if (cap < size) return ACO_ERR_CAPACITY;
        std::memcpy(tour, buf.data(), sizeof(int) * size);
    }
    return ACO_OK;
}

int aco_get_bsf_records(aco_solver *s, aco_record *out, int cap, int *count)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    int num = 0;
    CK(cudaMemcpyAsync(&num, s->d_num_bsf, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    const int stored = std::min(num, s->p.record_cap);
    if (count) *count = num;
    if (out && stored > 0) {
        CK(cudaMemcpyAsync(out, s->d_records, sizeof(aco_record) * std::min(stored, std::max(cap, 0)),
                           cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        if (cap < stored) return ACO_ERR_CAPACITY;
    }
    return ACO_OK;
}

int aco_get_solutions(aco_solver *s, int *solutions, size_t cap_ints, float *lens, size_t cap_lens)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const size_t ns = (size_t)s->T * (s->A + 1) + 1, nlens = (size_t)s->A + 1;
    if ((solutions && cap_ints < ns) || (lens && cap_lens < nlens)) return ACO_ERR_CAPACITY;
    if (solutions) CK(cudaMemcpyAsync(solutions, s->d_sol, ns * 4, cudaMemcpyDeviceToHost, s->st));
    if (lens) CK(cudaMemcpyAsync(lens, s->d_lens, nlens * 4, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ACO_OK;
}

int aco_get_pheromone(aco_solver *s, float *tau, float *total_info, size_t cap)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const size_t nn = (size_t)s->n * s->n;
    if (cap < nn) return ACO_ERR_CAPACITY;
    const size_t w = (size_t)s->n * 4, pitch = (size_t)s->ld * 4;
    if (tau) CK(cudaMemcpy2DAsync(tau, w, s->d_tau, pitch, w, s->n, cudaMemcpyDeviceToHost, s->st));
    if (total_info) CK(cudaMemcpy2DAsync(total_info, w, s->d_total, pitch, w, s->n, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ACO_OK;
}

int aco_get_seeds(aco_solver *s, int *seeds, size_t cap)
{
    if (!s || !seeds) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const size_t ns = (size_t)s->A * s->nloc;
    if (cap < ns) return ACO_ERR_CAPACITY;
    CK(cudaMemcpyAsync(seeds, s->d_seeds, ns * 4, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ACO_OK;
}

int aco_get_elites(aco_solver *s, int *elites, int cap)
{
    if (!s || !elites) return ACO_ERR_INVALID;
    if (cap < s->R) return ACO_ERR_CAPACITY;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    CK(cudaMemcpyAsync(elites, s->d_elites, sizeof(int) * s->R, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ACO_OK;
}

int aco_get_iteration(aco_solver *s, int *iteration)
{
    if (!s || !iteration) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    CK(cudaMemcpyAsync(s->h_pin + 1, s->d_iter, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    *iteration = s->h_pin[1];
    return ACO_OK;
}

int aco_set_state(aco_solver *s, const float *tau, const float *total_info, const int *solutions, const float *lens,
                  const int *seeds)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    const size_t w = (size_t)s->n * 4, pitch = (size_t)s->ld * 4;
    if (tau) CK(cudaMemcpy2DAsync(s->d_tau, pitch, tau, w, w, s->n, cudaMemcpyHostToDevice, s->st));
    if (total_info) CK(cudaMemcpy2DAsync(s->d_total, pitch, total_info, w, w, s->n, cudaMemcpyHostToDevice, s->st));
    if (solutions)
        CK(cudaMemcpyAsync(s->d_sol, solutions, ((size_t)s->T * (s->A + 1) + 1) * 4, cudaMemcpyHostToDevice, s->st));
    if (lens) CK(cudaMemcpyAsync(s->d_lens, lens, ((size_t)s->A + 1) * 4, cudaMemcpyHostToDevice, s->st));
    if (seeds) CK(cudaMemcpyAsync(s->d_seeds, seeds, (size_t)s->A * s->nloc * 4, cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->initialized = true;
    return ACO_OK;
}

int aco_status(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (set_device(s) != ACO_OK) return ACO_ERR_CUDA;
    return sync_status(s);
}

const char *aco_strerror(int code)
{
    switch (code) {
    case ACO_OK: return "ok";
    case ACO_ERR_INVALID: return "invalid argument";
    case ACO_ERR_INFEASIBLE: return "infeasible instance: a customer can never be served";
    case ACO_ERR_CUDA: return "CUDA runtime error";
    case ACO_ERR_NO_DEVICE: return "no usable sm_100 device";
    case ACO_ERR_NOMEM: return "out of memory";
    case ACO_ERR_STATE: return "call out of order";
    case ACO_ERR_STEP_LIMIT: return "construction exceeded its step budget";
    case ACO_ERR_LS_LIMIT: return "2-opt exceeded its pass budget";
    case ACO_ERR_RECORD_OVERFLOW: return "best-so-far record buffer full";
    case ACO_ERR_CAPACITY: return "output buffer too small";
    case ACO_ERR_IO: return "instance file missing or malformed";
    case ACO_ERR_TIMEOUT: return "a bounded device wait gave up";
    default: return "unknown error";
    }
}

void *aco_get_stream(aco_solver *s) { return s ? (void *)s->st : nullptr; }

int aco_launches_per_iteration(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    return 3 + (s->p.ls_flag ? 1 : 0);
}

int aco_time_iterations(aco_solver *s, int n_iter, float *ms)
{
    if (!s || !ms || n_iter <= 0) return ACO_ERR_INVALID;
    if (!s->initialized) return ACO_ERR_STATE;
    int rc = set_device(s);
    if (rc != ACO_OK) return rc;
    if (s->p.use_graph) {
        rc = ensure_graph(s);
        if (rc != ACO_OK) return rc;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s->st));
    for (int i = 0; i < n_iter && rc == ACO_OK; i++) {
        if (s->p.use_graph) {
            if (cudaGraphLaunch(s->exec, s->st) != cudaSuccess) rc = ACO_ERR_CUDA;
        } else {
            rc = run_iteration_phases(s);
        }
    }
    CK(cudaEventRecord(e1, s->st));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != ACO_OK) return rc;
    return sync_status(s);
}

int aco_enqueue_iterations(aco_solver *s, int n_iter)
{
    if (!s || n_iter < 0) return ACO_ERR_INVALID;
    if (!s->initialized) return ACO_ERR_STATE;
    int rc = set_device(s);
    if (rc != ACO_OK) return rc;
    if (s->p.use_graph) {
        rc = ensure_graph(s);
        if (rc != ACO_OK) return rc;
        for (int i = 0; i < n_iter; i++) CK(cudaGraphLaunch(s->exec, s->st));
        return ACO_OK;
    }
    for (int i = 0; i < n_iter && rc == ACO_OK; i++) rc = run_iteration_phases(s);
    return rc;
}

int aco_time_phases(aco_solver *s, int n_iter, float *ms4)
{
    if (!s || !ms4 || n_iter <= 0) return ACO_ERR_INVALID;
    if (!s->initialized) return ACO_ERR_STATE;
    int rc = set_device(s);
    if (rc != ACO_OK) return rc;
    cudaEvent_t ev[5];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    for (int k = 0; k < 4; k++) ms4[k] = 0.f;
    for (int it = 0; it < n_iter && rc == ACO_OK; it++) {
        CK(cudaEventRecord(ev[0], s->st));
        rc = do_construct(s);
        CK(cudaEventRecord(ev[1], s->st));
        if (rc == ACO_OK && s->p.ls_flag) rc = do_local_search(s);
        CK(cudaEventRecord(ev[2], s->st));
        if (rc == ACO_OK) rc = do_stats(s, true);
        CK(cudaEventRecord(ev[3], s->st));
        if (rc == ACO_OK) rc = do_update(s);
        CK(cudaEventRecord(ev[4], s->st));
        CK(cudaEventSynchronize(ev[4]));
        for (int k = 0; k < 4; k++) {
            float m = 0.f;
            CK(cudaEventElapsedTime(&m, ev[k], ev[k + 1]));
            ms4[k] += m;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc != ACO_OK) return rc;
    return sync_status(s);
}

int aco_get_config(aco_solver *s, int *ants_per_block, int *warps_per_ant, int *staging_flags)
{
    if (!s) return ACO_ERR_INVALID;
    const bool thr = s->p.mode == ACO_MODE_THROUGHPUT;
    if (ants_per_block) *ants_per_block = thr ? s->cn_apc : s->cp_apc;
    if (warps_per_ant) *warps_per_ant = thr ? 1 : s->cp_wpa;
    if (staging_flags) *staging_flags = ((thr ? s->cn_stage : s->cp_stage) ? 1 : 0) | (s->ls_snn ? 2 : 0);
    return ACO_OK;
}

} // extern "C"
