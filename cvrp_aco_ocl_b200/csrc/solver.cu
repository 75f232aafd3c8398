// solver.cu -- the C ABI of include/cvrp_aco.h: g_ACO's lifecycle
// (cvrp_ocl/gpu/g_aco.cpp) on one CUDA stream of one B200.
//
// aco_create   = g_ACO::g_ACO + create_memory_objects (g_aco.cpp:35-43, 640-761)
// aco_init     = g_ACO::init_aco (g_aco.cpp:63-93)
// aco_iterate  = run_aco_iteration (g_aco.cpp:122-134) + iteration++ (main.cpp:86),
//                replayed as one CUDA graph of four kernels:
//                construct -> 2-opt -> stats (best, bsf, elites, deposit list)
//                -> fused evaporation/deposit/total_info pass.
// A solver is a colony of one instance (colony.h); aco_batch_* drives a colony
// of many independent instances with the same launches.  All state stays on
// the device; the host synchronises once per aco_iterate call and reads a
// 4-byte status word.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/cvrp_aco.h"
#include "colony.h"
#include "host.h"
#include "kernels.h"

using namespace aco;

// Pipelined length readback: a ring of pinned host slots, each filled by a
// stream-ordered copy and marked by an event, so a caller can queue the next
// iteration before waiting for the lengths of the previous one.
constexpr int kLenSlots = 4;

// The ring of one colony: slot k holds `words` lengths and the status word.
struct LenRing {
    float *ring = nullptr;
    int words = 0;
    cudaEvent_t ev[kLenSlots] = {};
    long long ticket[kLenSlots] = {-1, -1, -1, -1};
    long long next = 0;
    void release(Colony &c)
    {
        if (!ring) return;
        c.set_device();
        cudaStreamSynchronize(c.st);
        for (int k = 0; k < kLenSlots; k++)
            if (ev[k]) cudaEventDestroy(ev[k]);
        cudaFreeHost(ring);
        ring = nullptr;
    }
};

struct aco_solver {
    Colony c;
    LenRing lr; // A + 1 lengths per slot
    ~aco_solver() { lr.release(c); }
};

struct aco_batch {
    Colony c;
    LenRing lr; // every instance's A + 1 lengths per slot (the colony's contiguous block)
    ~aco_batch() { lr.release(c); }
};

namespace {

#define CK(x)                                                                                                  \
    do {                                                                                                       \
        cudaError_t e_ = (x);                                                                                  \
        if (e_ != cudaSuccess) {                                                                               \
            aco::note_cuda_error(e_);                                                                          \
            return ACO_ERR_CUDA;                                                                               \
        }                                                                                                      \
    } while (0)

// Parameter checks shared by aco_create and aco_batch_create.
int check_params(const aco_params &p, int n)
{
    if (p.nloc < 32 || p.nloc > 1024 || (p.nloc & (p.nloc - 1))) return ACO_ERR_INVALID;
    if (p.ras_ranks < 1 || p.ras_ranks > 32) return ACO_ERR_INVALID;
    if (p.nn_ls < 0 || p.nn_ls > n - 2) return ACO_ERR_INVALID; // depth n-1 would list the node itself
    if (p.mode != ACO_MODE_PARITY && p.mode != ACO_MODE_THROUGHPUT) return ACO_ERR_INVALID;
    if (p.mode == ACO_MODE_THROUGHPUT && (p.nn_ants < 1 || p.nn_ants > 32 || p.nn_ants > n - 2))
        return ACO_ERR_INVALID;
    if (p.warps_per_ant != 0 && (p.warps_per_ant < 1 || p.warps_per_ant > 8 ||
                                 (p.warps_per_ant & (p.warps_per_ant - 1)) || 32 * p.warps_per_ant > p.nloc))
        return ACO_ERR_INVALID;
    if (p.ants_per_block < 0 || p.ants_per_block > 16) return ACO_ERR_INVALID;
    if (p.ls_warps < 0 || p.ls_warps > 32) return ACO_ERR_INVALID;
    if (p.stage_matrix < -1 || p.stage_matrix > 0) return ACO_ERR_INVALID;
    if (p.host_prep < 0 || p.host_prep > 1) return ACO_ERR_INVALID;
    if (p.ls_flag != 0 && p.ls_flag != 1 && p.ls_flag != 3) return ACO_ERR_INVALID;
    if (p.ns_rounds < 0 || p.ns_rounds > 1000000) return ACO_ERR_INVALID;
    if (p.fuse_ls < 0 || p.fuse_ls > 1) return ACO_ERR_INVALID;
    if (p.ls_ants < 0 || p.ls_ants > 8) return ACO_ERR_INVALID;
    if (p.draw_warps < -1 || p.draw_warps > 1) return ACO_ERR_INVALID;
    if (p.route_ls < -1 || p.route_ls > 1) return ACO_ERR_INVALID;
    if (p.wait_limit < 0) return ACO_ERR_INVALID;
    if (p.ls_best < 0 || p.ls_best > 1) return ACO_ERR_INVALID;
    if (p.construct_ctas < 0 || p.construct_ctas > 2) return ACO_ERR_INVALID;
    if (!(p.rho > 0.0f && p.rho <= 1.0f)) return ACO_ERR_INVALID;
    if (p.n_ants > 56 * 1024) return ACO_ERR_INVALID; // the statistics kernel holds n_ants lengths in shared memory
    return ACO_OK;
}

InstanceSpec spec_of(const aco_instance &in)
{
    InstanceSpec sp;
    sp.n = in.n;
    sp.x = in.x;
    sp.y = in.y;
    sp.demand = in.demand;
    sp.capacity = in.capacity;
    sp.max_dist = in.max_distance;
    sp.serv_time = in.service_time;
    sp.dist_type = in.dist_type;
    sp.dist = in.dist;
    return sp;
}

bool spec_ok(const aco_instance &in)
{
    return in.n >= 3 && in.n <= 32767 && in.demand && (in.dist || (in.x && in.y));
}

// Device-to-host copy of the reference-layout buffers of instance b.
int copy_solutions(Colony &c, int b, int *solutions, size_t cap_ints, float *lens, size_t cap_lens)
{
    const InstHost &ih = c.inst[b];
    const size_t ns = (size_t)ih.T * (ih.A + 1) + 1, nlens = (size_t)ih.A + 1;
    if ((solutions && cap_ints < ns) || (lens && cap_lens < nlens)) return ACO_ERR_CAPACITY;
    if (solutions) CK(cudaMemcpyAsync(solutions, ih.sol_d, ns * 4, cudaMemcpyDeviceToHost, c.st));
    if (lens) CK(cudaMemcpyAsync(lens, ih.lens_d, nlens * 4, cudaMemcpyDeviceToHost, c.st));
    CK(cudaStreamSynchronize(c.st));
    return ACO_OK;
}

int copy_best(Colony &c, int b, int *tour, int cap, int *tour_size, float *length)
{
    const InstHost &ih = c.inst[b];
    std::vector<int> buf(ih.T);
    float len = 0;
    CK(cudaMemcpyAsync(buf.data(), ih.sol_d + (size_t)ih.T * ih.A, sizeof(int) * ih.T, cudaMemcpyDeviceToHost, c.st));
    CK(cudaMemcpyAsync(&len, ih.lens_d + ih.A, sizeof(float), cudaMemcpyDeviceToHost, c.st));
    CK(cudaStreamSynchronize(c.st));
    const int size = buf[ih.T - 1];
    if (tour_size) *tour_size = size;
    if (length) *length = len;
    if (tour) {
        if (cap < size) return ACO_ERR_CAPACITY;
        std::memcpy(tour, buf.data(), sizeof(int) * size);
    }
    return ACO_OK;
}

int copy_pheromone(Colony &c, int b, float *tau, float *total_info, size_t cap)
{
    const InstHost &ih = c.inst[b];
    const size_t nn = (size_t)ih.n * ih.n;
    if (cap < nn) return ACO_ERR_CAPACITY;
    const size_t w = (size_t)ih.n * 4, pitch = (size_t)ih.ld * 4;
    if (tau) CK(cudaMemcpy2DAsync(tau, w, ih.tau_d, pitch, w, ih.n, cudaMemcpyDeviceToHost, c.st));
    if (total_info) CK(cudaMemcpy2DAsync(total_info, w, ih.total_d, pitch, w, ih.n, cudaMemcpyDeviceToHost, c.st));
    CK(cudaStreamSynchronize(c.st));
    return ACO_OK;
}

int copy_records(Colony &c, int b, aco_record *out, int cap, int *count)
{
    const InstHost &ih = c.inst[b];
    int num = 0;
    CK(cudaMemcpyAsync(&num, ih.nbsf_d, sizeof(int), cudaMemcpyDeviceToHost, c.st));
    CK(cudaStreamSynchronize(c.st));
    const int stored = std::min(num, c.p.record_cap);
    if (count) *count = num;
    if (out && stored > 0) {
        CK(cudaMemcpyAsync(out, ih.rec_d, sizeof(aco_record) * std::min(stored, std::max(cap, 0)),
                           cudaMemcpyDeviceToHost, c.st));
        CK(cudaStreamSynchronize(c.st));
        if (cap < stored) return ACO_ERR_CAPACITY;
    }
    return ACO_OK;
}

int run_sync(Colony &c, int rc) { return rc != ACO_OK ? rc : c.sync_status(); }

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

const char *aco_last_cuda_error(void)
{
    const cudaError_t e = last_cuda_error();
    return e == cudaSuccess ? "no error" : cudaGetErrorString(e);
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

int aco_create(const aco_instance *inst, const aco_params *params, aco_solver **out)
{
    if (!inst || !out || !inst->demand) return ACO_ERR_INVALID;
    *out = nullptr;
    const int n = inst->n;
    if (n < 2 || n > 32767) return ACO_ERR_INVALID;
    if (!inst->dist && (!inst->x || !inst->y)) return ACO_ERR_INVALID;
    aco_params p;
    if (params) p = *params;
    else aco_params_default(&p, n);
    if (p.n_ants <= 0) p.n_ants = n;
    if (p.record_cap <= 0) p.record_cap = 4096;
    int rc = check_params(p, n);
    if (rc != ACO_OK) return rc;
    aco_solver *s = new (std::nothrow) aco_solver;
    if (!s) return ACO_ERR_NOMEM;
    const InstanceSpec sp = spec_of(*inst);
    rc = s->c.create(&sp, 1, p);
    if (rc != ACO_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return ACO_OK;
}

void aco_destroy(aco_solver *s) { delete s; }

int aco_init(aco_solver *s) { return s ? s->c.init() : ACO_ERR_INVALID; }

int aco_iterate(aco_solver *s, int n_iter)
{
    if (!s || n_iter < 0) return ACO_ERR_INVALID;
    return run_sync(s->c, s->c.enqueue(n_iter));
}

int aco_clear_status(aco_solver *s) { return s ? s->c.clear_status() : ACO_ERR_INVALID; }

int aco_set_wait_limit(aco_solver *s, int polls) { return s ? s->c.set_wait_limit(polls) : ACO_ERR_INVALID; }

int aco_enqueue_iterations(aco_solver *s, int n_iter)
{
    if (!s || n_iter < 0) return ACO_ERR_INVALID;
    return s->c.enqueue(n_iter);
}

namespace {
// Queue a copy of `words` floats from `src` (and the status word) into the
// next ring slot; the ticket names the slot's copy.
int ring_enqueue(Colony &c, LenRing &lr, const float *src, int words, long long *ticket)
{
    if (!c.initialized) return ACO_ERR_STATE;
    if (c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    if (!lr.ring) { // first use: the ring and its events
        if (cudaMallocHost(&lr.ring, sizeof(float) * (size_t)(words + 1) * kLenSlots) != cudaSuccess) {
            lr.ring = nullptr;
            return ACO_ERR_NOMEM;
        }
        lr.words = words;
        for (int k = 0; k < kLenSlots; k++) CK(cudaEventCreateWithFlags(&lr.ev[k], cudaEventDisableTiming));
    }
    const long long t = lr.next;
    const int slot = (int)(t % kLenSlots);
    float *dst = lr.ring + (size_t)slot * (words + 1);
    CK(cudaMemcpyAsync(dst, src, sizeof(float) * words, cudaMemcpyDeviceToHost, c.st));
    CK(cudaMemcpyAsync(dst + words, c.status_d, sizeof(int), cudaMemcpyDeviceToHost, c.st));
    CK(cudaEventRecord(lr.ev[slot], c.st));
    lr.ticket[slot] = t;
    lr.next = t + 1;
    *ticket = t;
    return ACO_OK;
}

int ring_read(Colony &c, LenRing &lr, long long ticket, float *lens, size_t cap)
{
    const int slot = (int)(ticket % kLenSlots);
    if (!lr.ring || lr.ticket[slot] != ticket) return ACO_ERR_STATE; // never queued, or overwritten
    if (cap < (size_t)lr.words) return ACO_ERR_CAPACITY;
    if (c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    CK(cudaEventSynchronize(lr.ev[slot]));
    const float *src = lr.ring + (size_t)slot * (lr.words + 1);
    std::memcpy(lens, src, sizeof(float) * lr.words);
    int status;
    std::memcpy(&status, src + lr.words, sizeof(int));
    return status; // the device status word when the copy was queued
}

// The launch shape a colony planned (aco_get_config, aco_batch_get_config).
int get_config(const Colony &c, int *ants_per_block, int *warps_per_ant, int *staging_flags)
{
    const bool thr = c.p.mode == ACO_MODE_THROUGHPUT;
    if (ants_per_block) *ants_per_block = thr ? c.cn_apc : c.cp_apc;
    if (warps_per_ant) *warps_per_ant = thr ? 1 : c.cp_wpa;
    if (staging_flags)
        *staging_flags = (thr ? (c.inst[0].smat ? 1 : 0) : (c.cp_stage ? 1 : 0)) | 2 | (thr && c.cn_draw ? 4 : 0) |
                         (thr && c.cn_wide && c.cn_lsw == 0 ? 8 : 0);
    return ACO_OK;
}

} // namespace

int aco_enqueue_lengths(aco_solver *s, long long *ticket)
{
    if (!s || !ticket) return ACO_ERR_INVALID;
    return ring_enqueue(s->c, s->lr, s->c.inst[0].lens_d, s->c.inst[0].A + 1, ticket);
}

int aco_read_lengths(aco_solver *s, long long ticket, float *lens, size_t cap)
{
    if (!s || !lens || ticket < 0) return ACO_ERR_INVALID;
    return ring_read(s->c, s->lr, ticket, lens, cap);
}

int aco_batch_enqueue_lengths(aco_batch *b, long long *ticket)
{
    if (!b || !ticket) return ACO_ERR_INVALID;
    return ring_enqueue(b->c, b->lr, b->c.lens_all(), b->c.lens_total(), ticket);
}

int aco_batch_read_lengths(aco_batch *b, long long ticket, float *lens, size_t cap)
{
    if (!b || !lens || ticket < 0) return ACO_ERR_INVALID;
    return ring_read(b->c, b->lr, ticket, lens, cap);
}

int aco_batch_get_best_all(aco_batch *b, int *tours, size_t cap_ints, int *tour_sizes, float *lengths)
{
    if (!b) return ACO_ERR_INVALID;
    if (!b->c.initialized) return ACO_ERR_STATE;
    return b->c.get_best_all(tours, cap_ints, tour_sizes, lengths);
}

int aco_run(aco_solver *s, float optimum, int *iterations_done)
{
    if (!s) return ACO_ERR_INVALID;
    Colony &c = s->c;
    int rc = ACO_OK;
    if (!c.initialized) {
        rc = c.init();
        if (rc != ACO_OK) return rc;
    }
    const InstHost &ih = c.inst[0];
    int done = 0;
    for (;;) { // termination_condition (main.cpp:29-34)
        CK(cudaMemcpyAsync(c.h_pin + 1, ih.iter_d, sizeof(int), cudaMemcpyDeviceToHost, c.st));
        CK(cudaMemcpyAsync(c.h_pin + 2, ih.lens_d + ih.A, sizeof(float), cudaMemcpyDeviceToHost, c.st));
        CK(cudaStreamSynchronize(c.st));
        const int it = c.h_pin[1];
        float best = 0;
        std::memcpy(&best, c.h_pin + 2, sizeof(float));
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - c.t_init).count();
        if (it >= c.p.max_iteration || el >= c.p.max_runtime || std::fabs(best - optimum) < 10 * kEpsilon) break;
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
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return run_sync(s->c, s->c.construct());
}

int aco_local_search(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return run_sync(s->c, s->c.local_search());
}

int aco_update_statistics(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return run_sync(s->c, s->c.stats(true));
}

int aco_pheromone_update(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return run_sync(s->c, s->c.update());
}

int aco_pheromone_init(aco_solver *s, float trail_0)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return run_sync(s->c, s->c.pheromone_init(trail_0, false));
}

int aco_get_best(aco_solver *s, int *tour, int cap, int *tour_size, float *length)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_best(s->c, 0, tour, cap, tour_size, length);
}

int aco_get_bsf_records(aco_solver *s, aco_record *out, int cap, int *count)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_records(s->c, 0, out, cap, count);
}

int aco_get_solutions(aco_solver *s, int *solutions, size_t cap_ints, float *lens, size_t cap_lens)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_solutions(s->c, 0, solutions, cap_ints, lens, cap_lens);
}

int aco_get_pheromone(aco_solver *s, float *tau, float *total_info, size_t cap)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_pheromone(s->c, 0, tau, total_info, cap);
}

int aco_get_seeds(aco_solver *s, int *seeds, size_t cap)
{
    if (!s || !seeds) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    const InstHost &ih = s->c.inst[0];
    const size_t ns = (size_t)ih.A * ih.nloc;
    if (cap < ns) return ACO_ERR_CAPACITY;
    CK(cudaMemcpyAsync(seeds, ih.seeds_d, ns * 4, cudaMemcpyDeviceToHost, s->c.st));
    CK(cudaStreamSynchronize(s->c.st));
    return ACO_OK;
}

int aco_get_elites(aco_solver *s, int *elites, int cap)
{
    if (!s || !elites) return ACO_ERR_INVALID;
    const InstHost &ih = s->c.inst[0];
    if (cap < ih.R) return ACO_ERR_CAPACITY;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    CK(cudaMemcpyAsync(elites, ih.elites_d, sizeof(int) * ih.R, cudaMemcpyDeviceToHost, s->c.st));
    CK(cudaStreamSynchronize(s->c.st));
    return ACO_OK;
}

int aco_get_iteration(aco_solver *s, int *iteration)
{
    if (!s || !iteration) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    CK(cudaMemcpyAsync(s->c.h_pin + 1, s->c.inst[0].iter_d, sizeof(int), cudaMemcpyDeviceToHost, s->c.st));
    CK(cudaStreamSynchronize(s->c.st));
    *iteration = s->c.h_pin[1];
    return ACO_OK;
}

int aco_set_state(aco_solver *s, const float *tau, const float *total_info, const int *solutions, const float *lens,
                  const int *seeds)
{
    if (!s) return ACO_ERR_INVALID;
    Colony &c = s->c;
    if (c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    const InstHost &ih = c.inst[0];
    const size_t w = (size_t)ih.n * 4, pitch = (size_t)ih.ld * 4;
    if (tau) CK(cudaMemcpy2DAsync(ih.tau_d, pitch, tau, w, w, ih.n, cudaMemcpyHostToDevice, c.st));
    if (total_info) CK(cudaMemcpy2DAsync(ih.total_d, pitch, total_info, w, w, ih.n, cudaMemcpyHostToDevice, c.st));
    if (solutions)
        CK(cudaMemcpyAsync(ih.sol_d, solutions, ((size_t)ih.T * (ih.A + 1) + 1) * 4, cudaMemcpyHostToDevice, c.st));
    if (lens) CK(cudaMemcpyAsync(ih.lens_d, lens, ((size_t)ih.A + 1) * 4, cudaMemcpyHostToDevice, c.st));
    if (seeds) CK(cudaMemcpyAsync(ih.seeds_d, seeds, (size_t)ih.A * ih.nloc * 4, cudaMemcpyHostToDevice, c.st));
    if (total_info) {
        const int rc = c.gather_candidates(); // the construct kernel reads the candidates' total_info
        if (rc != ACO_OK) return rc;
    }
    CK(cudaStreamSynchronize(c.st));
    c.initialized = true;
    return ACO_OK;
}

int aco_status(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return s->c.sync_status();
}

void *aco_get_stream(aco_solver *s) { return s ? (void *)s->c.st : nullptr; }

int aco_launches_per_iteration(aco_solver *s)
{
    if (!s) return ACO_ERR_INVALID;
    return s->c.launches_per_iteration();
}

int aco_batch_launches_per_iteration(aco_batch *b)
{
    if (!b) return ACO_ERR_INVALID;
    return b->c.launches_per_iteration();
}

int aco_time_iterations(aco_solver *s, int n_iter, float *ms)
{
    if (!s || !ms || n_iter <= 0) return ACO_ERR_INVALID;
    Colony &c = s->c;
    if (!c.initialized) return ACO_ERR_STATE;
    if (c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    int rc = c.enqueue(0); // builds the graph outside the timed region
    if (rc != ACO_OK) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c.st));
    rc = c.enqueue(n_iter);
    CK(cudaEventRecord(e1, c.st));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return run_sync(c, rc);
}

int aco_time_phases(aco_solver *s, int n_iter, float *ms4)
{
    if (!s || !ms4 || n_iter <= 0) return ACO_ERR_INVALID;
    return s->c.time_phases(n_iter, ms4);
}

int aco_get_config(aco_solver *s, int *ants_per_block, int *warps_per_ant, int *staging_flags)
{
    return s ? get_config(s->c, ants_per_block, warps_per_ant, staging_flags) : ACO_ERR_INVALID;
}

int aco_batch_get_config(aco_batch *b, int *ants_per_block, int *warps_per_ant, int *staging_flags)
{
    return b ? get_config(b->c, ants_per_block, warps_per_ant, staging_flags) : ACO_ERR_INVALID;
}


int aco_validate(aco_solver *s, int *flags, int *n_invalid)
{
    if (!s) return ACO_ERR_INVALID;
    return s->c.validate(flags, nullptr, n_invalid);
}

namespace {
// The reference's solution block (io.cpp:270-281) for one tour.
void write_block(FILE *f, const int *tour, int size, float length)
{
    std::fprintf(f, "Begin Solution\n");
    for (int i = 0; i < size; i++) std::fprintf(f, "%d ", tour[i]);
    std::fprintf(f, "\nSolution Length %f\nEnd Solution\n", length);
}

int write_best(Colony &c, const char *path, bool batch)
{
    if (!path) return ACO_ERR_INVALID;
    FILE *f = std::fopen(path, "w");
    if (!f) return ACO_ERR_IO;
    int rc = ACO_OK;
    for (int b = 0; b < (int)c.inst.size() && rc == ACO_OK; b++) {
        std::vector<int> tour(c.inst[b].T);
        int size = 0;
        float len = 0.f;
        rc = copy_best(c, b, tour.data(), (int)tour.size(), &size, &len);
        if (rc != ACO_OK) break;
        if (batch) std::fprintf(f, "Instance %d\n", b);
        write_block(f, tour.data(), size, len);
    }
    if (std::fclose(f) != 0 && rc == ACO_OK) rc = ACO_ERR_IO;
    return rc;
}
} // namespace

int aco_write_solution(aco_solver *s, const char *path)
{
    if (!s) return ACO_ERR_INVALID;
    if (s->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return write_best(s->c, path, false);
}

int aco_save_checkpoint(aco_solver *s, const char *path) { return s ? s->c.save_checkpoint(path) : ACO_ERR_INVALID; }

int aco_load_checkpoint(aco_solver *s, const char *path) { return s ? s->c.load_checkpoint(path) : ACO_ERR_INVALID; }

int aco_set_prior(aco_solver *s, const float *prior, int ld)
{
    if (!s) return ACO_ERR_INVALID;
    return s->c.set_prior(0, prior, ld);
}

/* ---- batches ------------------------------------------------------------ */

int aco_batch_create(const aco_instance *insts, int count, const aco_params *params, aco_batch **out)
{
    if (!insts || !out || !params || count < 1 || count > 65535) return ACO_ERR_INVALID;
    *out = nullptr;
    aco_params p = *params;
    if (p.mode != ACO_MODE_THROUGHPUT) return ACO_ERR_INVALID; // the parity kernel serves one instance
    if (p.record_cap <= 0) p.record_cap = 4096;
    int n_min = INT_MAX;
    std::vector<InstanceSpec> specs(count);
    for (int b = 0; b < count; b++) {
        if (!spec_ok(insts[b])) return ACO_ERR_INVALID;
        n_min = std::min(n_min, insts[b].n);
        specs[b] = spec_of(insts[b]);
    }
    // lists deeper than the smallest instance allows are clamped per instance
    aco_params pc = p;
    pc.nn_ls = std::min(p.nn_ls, n_min - 2);
    pc.nn_ants = std::min(p.nn_ants, n_min - 2);
    int rc = check_params(pc, n_min);
    if (rc != ACO_OK) return rc;
    if (p.n_ants <= 0) return ACO_ERR_INVALID;
    aco_batch *bt = new (std::nothrow) aco_batch;
    if (!bt) return ACO_ERR_NOMEM;
    rc = bt->c.create(specs.data(), count, p);
    if (rc != ACO_OK) {
        delete bt;
        return rc;
    }
    *out = bt;
    return ACO_OK;
}

void aco_batch_destroy(aco_batch *b) { delete b; }

int aco_batch_init(aco_batch *b) { return b ? b->c.init() : ACO_ERR_INVALID; }

int aco_batch_iterate(aco_batch *b, int n_iter)
{
    if (!b || n_iter < 0) return ACO_ERR_INVALID;
    return run_sync(b->c, b->c.enqueue(n_iter));
}

int aco_batch_enqueue_iterations(aco_batch *b, int n_iter)
{
    if (!b || n_iter < 0) return ACO_ERR_INVALID;
    return b->c.enqueue(n_iter);
}

int aco_batch_status(aco_batch *b)
{
    if (!b) return ACO_ERR_INVALID;
    if (b->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return b->c.sync_status();
}

int aco_batch_size(aco_batch *b, int *count, int *total_ants)
{
    if (!b) return ACO_ERR_INVALID;
    if (count) *count = (int)b->c.inst.size();
    if (total_ants) *total_ants = b->c.total_ants;
    return ACO_OK;
}

int aco_batch_get_best(aco_batch *b, int idx, int *tour, int cap, int *tour_size, float *length)
{
    if (!b || idx < 0 || idx >= (int)b->c.inst.size()) return ACO_ERR_INVALID;
    if (b->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_best(b->c, idx, tour, cap, tour_size, length);
}

int aco_batch_get_solutions(aco_batch *b, int idx, int *solutions, size_t cap_ints, float *lens, size_t cap_lens)
{
    if (!b || idx < 0 || idx >= (int)b->c.inst.size()) return ACO_ERR_INVALID;
    if (b->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_solutions(b->c, idx, solutions, cap_ints, lens, cap_lens);
}

int aco_batch_get_pheromone(aco_batch *b, int idx, float *tau, float *total_info, size_t cap)
{
    if (!b || idx < 0 || idx >= (int)b->c.inst.size()) return ACO_ERR_INVALID;
    if (b->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_pheromone(b->c, idx, tau, total_info, cap);
}

int aco_batch_time_phases(aco_batch *b, int n_iter, float *ms4)
{
    if (!b || !ms4 || n_iter <= 0) return ACO_ERR_INVALID;
    return b->c.time_phases(n_iter, ms4);
}

int aco_batch_save_checkpoint(aco_batch *b, const char *path)
{
    return b ? b->c.save_checkpoint(path) : ACO_ERR_INVALID;
}

int aco_batch_load_checkpoint(aco_batch *b, const char *path)
{
    return b ? b->c.load_checkpoint(path) : ACO_ERR_INVALID;
}

int aco_batch_validate(aco_batch *b, int *invalid_per_instance, int *n_invalid)
{
    if (!b) return ACO_ERR_INVALID;
    return b->c.validate(nullptr, invalid_per_instance, n_invalid);
}

int aco_batch_write_solutions(aco_batch *b, const char *path)
{
    if (!b) return ACO_ERR_INVALID;
    if (b->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return write_best(b->c, path, true);
}

int aco_batch_get_bsf_records(aco_batch *b, int idx, aco_record *out, int cap, int *count)
{
    if (!b || idx < 0 || idx >= (int)b->c.inst.size()) return ACO_ERR_INVALID;
    if (b->c.set_device() != ACO_OK) return ACO_ERR_CUDA;
    return copy_records(b->c, idx, out, cap, count);
}

int aco_batch_set_prior(aco_batch *b, int idx, const float *prior, int ld)
{
    if (!b) return ACO_ERR_INVALID;
    return b->c.set_prior(idx, prior, ld);
}

void *aco_batch_get_stream(aco_batch *b) { return b ? (void *)b->c.st : nullptr; }

} // extern "C"

/* ---- autotuner ------------------------------------------------------------ */

namespace {

// Per-kernel times (ms per iteration) of one configuration on a fresh colony.
int time_config(const InstanceSpec *specs, int count, const aco_params &p, int iters, float *ph4)
{
    Colony c;
    int rc = c.create(specs, count, p);
    if (rc == ACO_OK) rc = c.init();
    if (rc == ACO_OK) rc = c.enqueue(2);
    if (rc == ACO_OK) rc = c.sync_status();
    if (rc == ACO_OK) rc = c.time_phases(iters, ph4);
    if (rc != ACO_OK) return rc;
    for (int k = 0; k < 4; k++) ph4[k] /= (float)iters;
    return ACO_OK;
}

int autotune(const InstanceSpec *specs, int count, const aco_params &p0, int iters, aco_params *out, float *ms_out)
{
    if (iters < 1 || !out) return ACO_ERR_INVALID;
    const bool thr = p0.mode == ACO_MODE_THROUGHPUT;
    // The baseline is the configuration as given (its 0 fields chosen by the
    // create-time model); a candidate replaces it only when it is faster by more
    // than kMargin, so that timing noise does not pick a worse shape.
    constexpr float kMargin = 0.98f;
    // the per-ant 2-opt CTA shape: its time varies with the instance more than the margin
    constexpr float kMarginLs = 0.95f;
    aco_params best = p0;
    float best_ph[4] = {0, 0, 0, 0};
    float best_c = INFINITY;
    bool any = false;
    if (time_config(specs, count, p0, iters, best_ph) == ACO_OK) {
        best_c = best_ph[0] * kMargin;
        any = true;
    }
    // construct: ants per CTA x (warps per ant | matrix staging x (helper draw warps |
    // CTAs per SM))
    struct Cand {
        int apc, second, draw, ctas;
    };
    std::vector<Cand> cands;
    if (thr) {
        for (int apc : {1, 2, 4, 8, 16})
            for (int stage : {0, -1})
                for (int draw : {-1, 1}) {
                    if (p0.draw_warps != 0 && draw != p0.draw_warps) continue;
                    if (draw == 1 && apc > 8) continue; // a helper warp per ant: at most 8 ants per CTA
                    if (draw == 1) {
                        cands.push_back({apc, stage, draw, 1});
                        continue;
                    }
                    for (int ctas : {1, 2})
                        if (p0.construct_ctas == 0 || ctas == p0.construct_ctas) cands.push_back({apc, stage, draw, ctas});
                }
    } else {
        for (int wpa : {1, 2, 4, 8})
            for (int apc : {1, 2, 4, 8})
                if (wpa * apc <= 16 && 32 * wpa <= p0.nloc) cands.push_back({apc, wpa, 0, 0});
    }
    for (const auto &cd : cands) {
        aco_params q = p0;
        q.ants_per_block = cd.apc;
        if (thr) {
            q.stage_matrix = cd.second;
            q.draw_warps = cd.draw;
            q.construct_ctas = cd.ctas;
        } else {
            q.warps_per_ant = cd.second;
        }
        if (q.ls_warps == 0 && best.ls_warps != 0) q.ls_warps = best.ls_warps;
        float ph[4];
        if (time_config(specs, count, q, iters, ph) != ACO_OK) continue; // e.g. shared memory does not fit
        if (ph[0] < best_c) {
            best_c = ph[0] * kMargin;
            best = q;
            std::memcpy(best_ph, ph, sizeof(ph));
            any = true;
        }
    }
    if (!any) return ACO_ERR_INVALID;
    best_c = best_ph[0];
    // throughput mode: the route list (every route improved by one persistent kernel over
    // the SMs) against the per-ant kernel alone, with the chosen construct
    if (thr && (p0.ls_flag & 1) && p0.route_ls == 0) {
        int best_r = best.route_ls;
        float best_t = (best_ph[0] + best_ph[1]) * kMargin;
        for (int r : {-1, 1}) {
            aco_params q = best;
            q.route_ls = r;
            float ph[4];
            if (time_config(specs, count, q, iters, ph) != ACO_OK) continue;
            if (ph[0] + ph[1] < best_t) {
                best_t = (ph[0] + ph[1]) * kMargin;
                best_r = r;
                std::memcpy(best_ph, ph, sizeof(ph));
            }
        }
        best.route_ls = best_r;
        best_c = best_ph[0];
    }
    // 2-opt CTA shape (ants x warps) with the chosen construct; with the route
    // list the per-ant kernel only takes the ants the list does not hold
    if (p0.ls_flag && (p0.ls_warps == 0 || p0.ls_ants == 0) && best.route_ls != 1) {
        float best_l = best_ph[1] * kMarginLs;
        int best_a = p0.ls_ants, best_w = p0.ls_warps;
        for (int an : {1, 2, 4}) {
            if (p0.ls_ants != 0 && an != p0.ls_ants) continue;
            for (int w : {8, 12, 16, 24, 32}) {
                if (p0.ls_warps != 0 && w != p0.ls_warps) continue;
                if (w < an) continue;
                aco_params q = best;
                q.ls_ants = an;
                q.ls_warps = w;
                float ph[4];
                if (time_config(specs, count, q, iters, ph) != ACO_OK) continue;
                if (ph[1] < best_l) {
                    best_l = ph[1] * kMarginLs;
                    best_a = an;
                    best_w = w;
                    std::memcpy(best_ph, ph, sizeof(ph));
                    best_ph[0] = best_c;
                }
            }
        }
        best.ls_ants = best_a;
        best.ls_warps = best_w;
    }
    *out = best;
    if (ms_out) *ms_out = best_ph[0] + best_ph[1] + best_ph[2] + best_ph[3];
    return ACO_OK;
}

} // namespace

int aco_autotune(const aco_instance *inst, const aco_params *params, int iters, aco_params *out, float *ms_out)
{
    if (!inst || !out || !spec_ok(*inst)) return ACO_ERR_INVALID;
    const int n = inst->n;
    aco_params p;
    if (params) p = *params;
    else aco_params_default(&p, n);
    if (p.n_ants <= 0) p.n_ants = n;
    if (p.record_cap <= 0) p.record_cap = 4096;
    int rc = check_params(p, n);
    if (rc != ACO_OK) return rc;
    const InstanceSpec sp = spec_of(*inst);
    return autotune(&sp, 1, p, iters, out, ms_out);
}

int aco_batch_autotune(const aco_instance *insts, int count, const aco_params *params, int iters, aco_params *out,
                       float *ms_out)
{
    if (!insts || !params || !out || count < 1 || count > 65535) return ACO_ERR_INVALID;
    if (params->mode != ACO_MODE_THROUGHPUT || params->n_ants <= 0) return ACO_ERR_INVALID;
    std::vector<InstanceSpec> specs(count);
    int n_min = INT_MAX;
    for (int b = 0; b < count; b++) {
        if (!spec_ok(insts[b])) return ACO_ERR_INVALID;
        n_min = std::min(n_min, insts[b].n);
        specs[b] = spec_of(insts[b]);
    }
    aco_params pc = *params;
    pc.nn_ls = std::min(pc.nn_ls, n_min - 2);
    pc.nn_ants = std::min(pc.nn_ants, n_min - 2);
    const int rc = check_params(pc, n_min);
    if (rc != ACO_OK) return rc;
    aco_params p = *params;
    if (p.record_cap <= 0) p.record_cap = 4096;
    return autotune(specs.data(), count, p, iters, out, ms_out);
}
