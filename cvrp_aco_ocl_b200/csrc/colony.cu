// colony.cu -- host side of one ACO iteration over one or more instances:
// preprocessing (g_ACO::create_memory_objects, g_aco.cpp:640-761, and
// init_problem, problem.cpp:43-56), the device arena, the launch sequence of
// run_aco_iteration (g_aco.cpp:122-134) and its CUDA graph.
#include "colony.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>

#include "host.h"

namespace aco {

#define CK(x)                                                                                                  \
    do {                                                                                                       \
        cudaError_t e_ = (x);                                                                                  \
        if (e_ != cudaSuccess) {                                                                               \
            aco::note_cuda_error(e_);                                                                          \
            return ACO_ERR_CUDA;                                                                               \
        }                                                                                                      \
    } while (0)

namespace {

// 227 KB per CTA minus room for the kernels' static shared memory
constexpr size_t kSmemBudget = 226 * 1024;
// two construct CTAs per SM: 228 KB an SM, 1 KB of it reserved per CTA
constexpr size_t kWideBudget = 112 * 1024;
constexpr int kRouteWarps = 16; // warps per CTA of the route-level 2-opt
constexpr int kSwapLimitPerNode = 64; // accepted swaps per node and tour before ACO_ERR_LS_LIMIT

int exp_as_int(float e)
{
    if (e >= 0.0f && e <= 8.0f && e == (float)(int)e) return (int)e;
    return -1;
}

int ilog2(int v)
{
    int r = 0;
    while ((1 << r) < v) r++;
    return r;
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Uploads collected into one host blob; flush() copies it to a temporary
// device buffer in one transfer and scatters the pieces with one kernel.
struct Staging {
    std::vector<unsigned char> blob;
    std::vector<ScatterPiece> pieces;
    void add(void *dst, const void *src, size_t bytes)
    {
        if (bytes == 0) return;
        const size_t off = (blob.size() + 15) & ~(size_t)15;
        blob.resize(off + bytes);
        std::memcpy(blob.data() + off, src, bytes);
        pieces.push_back(ScatterPiece{(unsigned long long)(uintptr_t)dst, (unsigned long long)off,
                                      (unsigned long long)bytes});
    }
    cudaError_t flush(cudaMemPool_t pool, int sm_count, cudaStream_t st)
    {
        if (pieces.empty()) return cudaSuccess;
        const size_t poff = (blob.size() + 15) & ~(size_t)15;
        blob.resize(poff + pieces.size() * sizeof(ScatterPiece));
        std::memcpy(blob.data() + poff, pieces.data(), pieces.size() * sizeof(ScatterPiece));
        void *d = nullptr;
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&d, blob.size(), pool, st) : cudaMallocAsync(&d, blob.size(), st);
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(d, blob.data(), blob.size(), cudaMemcpyHostToDevice, st); // pageable: staged on return
        if (e == cudaSuccess)
            e = launch_scatter(reinterpret_cast<const ScatterPiece *>(static_cast<unsigned char *>(d) + poff),
                               (int)pieces.size(), static_cast<const unsigned char *>(d), poff, sm_count, st);
        const cudaError_t f = cudaFreeAsync(d, st);
        blob.clear();
        pieces.clear();
        return e != cudaSuccess ? e : f;
    }
};

// FNV-1a over bytes, continued from h.
uint64_t fnv1a(uint64_t h, const void *data, size_t bytes)
{
    const unsigned char *b = static_cast<const unsigned char *>(data);
    for (size_t k = 0; k < bytes; k++) {
        h ^= b[k];
        h *= 1099511628211ull;
    }
    return h;
}

constexpr uint64_t kFnvBasis = 14695981039346656037ull;

// Per-instance host preparation: distances, feasibility, NN lists.
int prep_instance(const InstanceSpec &sp, const aco_params &p, InstHost &ih)
{
    const int n = sp.n;
    {   // the instance's identity for checkpoints: its data as given
        uint64_t hh = fnv1a(kFnvBasis, &n, sizeof n);
        if (sp.x) hh = fnv1a(hh, sp.x, sizeof(float) * (size_t)n);
        if (sp.y) hh = fnv1a(hh, sp.y, sizeof(float) * (size_t)n);
        hh = fnv1a(hh, sp.demand, sizeof(int) * (size_t)n);
        if (sp.dist) hh = fnv1a(hh, sp.dist, sizeof(float) * (size_t)n * n);
        const float f[2] = {sp.max_dist, sp.serv_time};
        const int k[2] = {sp.capacity, sp.dist_type};
        hh = fnv1a(hh, f, sizeof f);
        ih.data_hash = fnv1a(hh, k, sizeof k);
    }
    ih.n = n;
    ih.ld = (n + 31) & ~31;
    ih.n4 = (n + 3) & ~3;
    ih.A = p.n_ants > 0 ? p.n_ants : n;
    ih.T = 2 * n;
    ih.K = p.mode == ACO_MODE_THROUGHPUT ? std::min(p.nn_ants, n - 2) : 0;
    if (ih.K < 0) ih.K = 0;
    ih.Kp = ih.K > 0 ? (ih.K + 7) & ~7 : 8;
    ih.nn_ls = std::max(0, std::min(p.nn_ls, n - 2));
    ih.R = p.ras_ranks;
    ih.nloc = p.nloc;
    ih.lg = ilog2(p.nloc);
    ih.kmax = (n + p.nloc - 1) / p.nloc;
    ih.capacity = sp.capacity;
    ih.max_dist = sp.max_dist;
    ih.serv_time = sp.serv_time;
    ih.demand.assign(sp.demand, sp.demand + n);
    ih.device_prep = !sp.dist && !p.host_prep && device_dist_supported(sp.dist_type) && nn_rows_per_cta(n) >= 1;
    ih.x = sp.x;
    ih.y = sp.y;
    ih.dist_type = sp.dist_type;
    if (!ih.device_prep) {
        ih.dist.resize((size_t)n * n);
        if (sp.dist) std::memcpy(ih.dist.data(), sp.dist, sizeof(float) * (size_t)n * n);
        else compute_distances(n, sp.x, sp.y, sp.dist_type, ih.dist.data());
    }
    for (int i = 1; i < n; i++) { // a customer nobody can serve makes construct loop forever (kernel.cl:438,461)
        if (ih.demand[i] > ih.capacity) return ACO_ERR_INFEASIBLE;
        if (std::isinf(ih.max_dist) && ih.max_dist > 0) continue;
        const float d0i = ih.device_prep ? point_distance(sp.x, sp.y, sp.dist_type, 0, i) : ih.dist[i];
        const float di0 = ih.device_prep ? point_distance(sp.x, sp.y, sp.dist_type, i, 0) : ih.dist[(size_t)i * n];
        const float reach = (0.0f + (d0i + ih.serv_time)) + di0;
        if (!(reach <= ih.max_dist)) return ACO_ERR_INFEASIBLE;
    }
    if (ih.device_prep) {
        int depth = std::max(ih.nn_ls, ih.K);
        if (depth >= n) depth = n - 1;
        ih.depth = std::max(depth, 0);
    } else {
        ih.depth = compute_nn_lists(n, ih.dist.data(), ih.nn_ls, ih.K, ih.nn);
    }
    return ACO_OK;
}

// Process-wide resources of one device, made once: its attributes, a memory
// pool for the colonies' arenas (freed blocks stay cached in the pool, so a
// new solver does not pay cudaMalloc's cost) and a block of pinned status
// words handed out in 64-byte slots.
struct DeviceRes {
    std::once_flag once;
    int rc = ACO_OK, sm = 0, major = 0;
    cudaMemPool_t pool = nullptr;
    int *pinned = nullptr;
    std::mutex mu;
    std::vector<int> free_slots;
    std::vector<cudaStream_t> free_streams; // streams of destroyed colonies, idle, reused by new ones
};

constexpr int kMaxDevices = 64, kSlotInts = 16, kSlots = 256;
DeviceRes g_res[kMaxDevices];

DeviceRes *device_res(int dev)
{
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    DeviceRes &r = g_res[dev];
    std::call_once(r.once, [&]() {
        int dc = 0;
        if (cudaGetDeviceCount(&dc) != cudaSuccess || dev >= dc) { r.rc = ACO_ERR_NO_DEVICE; return; }
        if (cudaDeviceGetAttribute(&r.major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&r.sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || r.major < 10) {
            r.rc = ACO_ERR_NO_DEVICE;
            return;
        }
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (cudaMemPoolCreate(&r.pool, &props) == cudaSuccess) {
            uint64_t keep = UINT64_MAX; // never hand cached blocks back to the driver
            cudaMemPoolSetAttribute(r.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            r.pool = nullptr;
        }
        if (cudaMallocHost(&r.pinned, sizeof(int) * kSlotInts * kSlots) == cudaSuccess) {
            for (int i = kSlots - 1; i >= 0; i--) r.free_slots.push_back(i);
        } else {
            r.pinned = nullptr;
        }
        cudaSetDevice(prev);
    });
    return &r;
}

int *take_pinned_slot(DeviceRes &r)
{
    std::lock_guard<std::mutex> lk(r.mu);
    if (!r.pinned || r.free_slots.empty()) return nullptr;
    const int i = r.free_slots.back();
    r.free_slots.pop_back();
    return r.pinned + (size_t)i * kSlotInts;
}

cudaStream_t take_stream(DeviceRes &r)
{
    std::lock_guard<std::mutex> lk(r.mu);
    if (r.free_streams.empty()) return nullptr;
    cudaStream_t s = r.free_streams.back();
    r.free_streams.pop_back();
    return s;
}

void give_stream(DeviceRes &r, cudaStream_t s)
{
    std::lock_guard<std::mutex> lk(r.mu);
    r.free_streams.push_back(s);
}

bool give_pinned_slot(DeviceRes &r, int *p)
{
    if (!r.pinned || p < r.pinned || p >= r.pinned + kSlotInts * kSlots) return false;
    std::lock_guard<std::mutex> lk(r.mu);
    r.free_slots.push_back((int)((p - r.pinned) / kSlotInts));
    return true;
}

} // namespace

namespace {
thread_local cudaError_t t_last_error = cudaSuccess;
}

void note_cuda_error(cudaError_t e) { t_last_error = e; }
cudaError_t last_cuda_error() { return t_last_error; }

Colony::~Colony()
{
    if (dev >= 0) cudaSetDevice(dev);
    if (st) cudaStreamSynchronize(st);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (void *q : allocs_) {
        if (pooled_ && st) cudaFreeAsync(q, st);
        else cudaFree(q);
    }
    if (st) cudaStreamSynchronize(st);
    DeviceRes *r = device_res(dev);
    if (h_pin && !(r && give_pinned_slot(*r, h_pin))) cudaFreeHost(h_pin);
    if (st) { // idle after the synchronisation above: kept for the next colony on this device
        if (r && cudaStreamQuery(st) == cudaSuccess) give_stream(*r, st);
        else cudaStreamDestroy(st);
    }
}

int Colony::set_device() const
{
    CK(cudaSetDevice(dev));
    return ACO_OK;
}

int Colony::create(const InstanceSpec *specs, int count, const aco_params &pin)
{
    p = pin;
    dev = p.device;
    inst.resize(count);
    // ---- host preparation, one thread per core over the instances
    {
        std::atomic<int> next{0}, err{ACO_OK};
        auto work = [&]() {
            for (;;) {
                const int b = next.fetch_add(1);
                if (b >= count) break;
                const int rc = prep_instance(specs[b], p, inst[b]);
                if (rc != ACO_OK) err.store(rc);
            }
        };
        const int nth = std::max(1, std::min<int>(count, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (int t = 1; t < nth; t++) th.emplace_back(work);
        work();
        for (auto &t : th) t.join();
        if (err.load() != ACO_OK) return err.load();
    }
    // ---- device
    DeviceRes *res = device_res(p.device);
    if (!res || res->rc != ACO_OK) return ACO_ERR_NO_DEVICE;
    sm_count = res->sm;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    st = take_stream(*res);
    if (!st) CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    h_pin = take_pinned_slot(*res);
    if (!h_pin) CK(cudaMallocHost(&h_pin, 64));

    // ---- arena layout
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = al256(off + std::max<size_t>(bytes, 16));
        return o;
    };
    struct Offs {
        size_t dist, heur, tau, total, chc, dem, key, jump, adv, cand32, nn16, nnls, seeds, sol, elites, succ,
            dep, dtau, rec, nbsf, iter, xy;
    };
    std::vector<Offs> offs(count);
    for (int b = 0; b < count; b++) {
        const InstHost &ih = inst[b];
        const size_t nl = (size_t)ih.n * ih.ld * 4;
        Offs &o = offs[b];
        o.dist = take(nl); o.heur = take(nl); o.tau = take(nl); o.total = take(nl);
        o.chc = take((size_t)ih.n * ih.Kp * 4);
        o.dem = take((size_t)ih.n4 * 4);
        o.key = take((size_t)ih.n4 * 4);
        o.jump = take((size_t)((ih.kmax + 3) & ~3) * 4);
        o.adv = take((size_t)ih.nloc * 4);
        o.cand32 = take((size_t)ih.n * ih.Kp * 4);
        o.nn16 = take((size_t)ih.n * ih.Kp * 2);
        o.nnls = take((size_t)ih.n * std::max(1, ih.nn_ls) * 4);
        o.seeds = take((size_t)ih.A * ih.nloc * 4);
        o.sol = take(((size_t)ih.T * (ih.A + 1) + 1) * 4);
        o.elites = take((size_t)ih.R * 4);
        o.succ = take((size_t)ih.R * ih.n * 4);
        o.dep = take((size_t)ih.n * 4);
        o.dtau = take((size_t)ih.R * 4);
        o.rec = take((size_t)p.record_cap * sizeof(aco_record));
        o.nbsf = take(4);
        o.iter = take(4);
        o.xy = ih.device_prep ? take((size_t)2 * ih.n4 * 4) : 0;
    }
    const size_t o_status = take(4), o_t0 = take(8), o_queue = take(8); // construct queue: next item, CTAs done
    const size_t o_wait = take(4); // poll limit of the device waits
    total_ants = 0;
    total_rows = 0;
    ld_max = 32;
    slot_base_h_.assign(count + 1, 0); // the lengths of all instances: one contiguous block
    tour_base_h_.assign(count + 1, 0); // the packed best-so-far tours of get_best_all
    for (int b = 0; b < count; b++) {
        const InstHost &ih = inst[b];
        total_ants += ih.A;
        total_rows += ih.n;
        ld_max = std::max(ld_max, ih.ld);
        slot_base_h_[b + 1] = slot_base_h_[b] + ih.A + 1;
        tour_base_h_[b + 1] = tour_base_h_[b] + ih.T;
    }
    const size_t o_lens_all = take((size_t)slot_base_h_[count] * 4);
    const size_t o_tour_base = take((size_t)(count + 1) * 4), o_best_tours = take((size_t)tour_base_h_[count] * 4);
    const size_t o_best_sizes = take((size_t)count * 4), o_best_lens = take((size_t)count * 4);
    const size_t o_ant_inst = take((size_t)total_ants * 4), o_ant_base = take((size_t)(count + 1) * 4);
    const size_t o_row_base = take((size_t)(count + 1) * 4), o_zero_base = take(16);
    const size_t o_row_inst = take((size_t)total_rows * 4); // instance of every global matrix row
    const size_t o_slot_base = take((size_t)(count + 1) * 4), o_valid = take((size_t)(total_ants + count) * 4);
    const size_t o_invalid = take((size_t)count * 4);
    const size_t o_cargs = take(sizeof(ConstructArgs) * count), o_largs = take(sizeof(LocalSearchArgs) * count);
    const size_t o_sargs = take(sizeof(StatsArgs) * count), o_uargs = take(sizeof(UpdateArgs) * count);
    const size_t o_pargs = take(sizeof(PrepArgs) * count);
    // construct work items {instance, first ant}, larger instances first
    // (set after cn_apc is known; sized for apc = 1)
    const size_t o_items = take((size_t)total_ants * sizeof(int2));
    const size_t o_sw_items = take((size_t)total_ants * sizeof(int2));
    const size_t o_ns_items = take((size_t)total_ants * sizeof(int2));
    const size_t o_ls_needed = take((size_t)total_ants);
    // route list of the route-level 2-opt: throughput mode with 2-opt, instances
    // whose distance matrix is symmetric (it sums tour lengths from the matrix)
    {
        int n_max = 0;
        bool sym = true;
        long long cap = 0;
        for (const InstHost &ih : inst) {
            n_max = std::max(n_max, ih.n);
            // routes per tour: at least total demand / capacity; twice that plus a margin,
            // and never more than one per customer
            long long dem = 0;
            for (int i = 1; i < ih.n; i++) dem += ih.demand[i];
            const long long per = ih.capacity > 0 ? 2 * ((dem + ih.capacity - 1) / ih.capacity) + 16 : ih.n - 1;
            cap += (long long)ih.A * std::min<long long>(ih.n - 1, per);
            if (!ih.device_prep) // coordinate formulas are symmetric; a given matrix is checked
                for (int i = 0; i < ih.n && sym; i++)
                    for (int j = 0; j < i; j++)
                        if (ih.dist[(size_t)i * ih.n + j] != ih.dist[(size_t)j * ih.n + i]) {
                            sym = false;
                            break;
                        }
        }
        // measured: with few ants per SM the per-ant kernel is as fast (the slowest
        // route sets the time either way) and the list costs the construct a pass
        use_routes_ = p.mode == ACO_MODE_THROUGHPUT && (p.ls_flag & 1) && sym && n_max <= 4096 &&
                      cap < (1ll << 30) && (p.route_ls > 0 || (p.route_ls == 0 && total_ants > 4 * sm_count));
        route_cap_ = use_routes_ ? (int)cap : 0;
    }
    const size_t o_rdesc = take((size_t)route_cap_ * sizeof(int2)), o_rctr = take(16);
    const size_t o_lslist = take((size_t)total_ants * 4), o_lsctr = take(16); // flagged ants for the per-ant 2-opt
    const size_t o_rrem = take((size_t)total_ants * 4);

    void *arena = nullptr;
    if (res->pool && cudaMallocFromPoolAsync(&arena, off, res->pool, st) == cudaSuccess) {
        pooled_ = true;
    } else {
        cudaGetLastError(); // clear a failed pool allocation before trying the plain one
        if (cudaMalloc(&arena, off) != cudaSuccess) return ACO_ERR_NOMEM;
    }
    allocs_.push_back(arena);
    arena_ = arena;
    CK(cudaMemsetAsync(arena, 0, off, st));
    char *base = static_cast<char *>(arena);
    for (int b = 0; b < count; b++) {
        InstHost &ih = inst[b];
        const Offs &o = offs[b];
        ih.dist_d = (float *)(base + o.dist); ih.heur_d = (float *)(base + o.heur);
        ih.tau_d = (float *)(base + o.tau); ih.total_d = (float *)(base + o.total);
        ih.chc_d = (float *)(base + o.chc); ih.dem_d = (int *)(base + o.dem);
        ih.key_d = (uint32_t *)(base + o.key); ih.jump_d = (uint32_t *)(base + o.jump);
        ih.adv_d = (uint32_t *)(base + o.adv); ih.cand32_d = (uint32_t *)(base + o.cand32);
        ih.nn16_d = (uint16_t *)(base + o.nn16); ih.nnls_d = (int *)(base + o.nnls);
        ih.seeds_d = (int *)(base + o.seeds); ih.sol_d = (int *)(base + o.sol);
        ih.lens_d = (float *)(base + o_lens_all) + slot_base_h_[b]; ih.elites_d = (int *)(base + o.elites);
        ih.succ_d = (int *)(base + o.succ); ih.dep_d = (uint32_t *)(base + o.dep);
        ih.dtau_d = (float *)(base + o.dtau); ih.rec_d = (aco_record *)(base + o.rec);
        ih.nbsf_d = (int *)(base + o.nbsf); ih.iter_d = (int *)(base + o.iter);
        if (ih.device_prep) {
            ih.xy_d = (float *)(base + o.xy);
        }
    }
    status_d = (int *)(base + o_status);
    wait_d = (int *)(base + o_wait);
    lens_all_d_ = (float *)(base + o_lens_all);
    tour_base_d_ = (int *)(base + o_tour_base);
    best_tours_d_ = (int *)(base + o_best_tours);
    best_sizes_d_ = (int *)(base + o_best_sizes);
    best_lens_d_ = (float *)(base + o_best_lens);
    t0_d_ = (unsigned long long *)(base + o_t0);
    queue_d_ = (int *)(base + o_queue);
    ant_inst_d_ = (int *)(base + o_ant_inst);
    ant_base_d_ = (int *)(base + o_ant_base);
    row_base_d_ = (int *)(base + o_row_base);
    row_inst_d_ = (int *)(base + o_row_inst);
    zero_base_d_ = (int *)(base + o_zero_base); // {0}: row base of a one-instance launch
    slot_base_d_ = (int *)(base + o_slot_base);
    valid_d_ = (int *)(base + o_valid);
    invalid_d_ = (int *)(base + o_invalid);
    cargs_d_ = (ConstructArgs *)(base + o_cargs);
    largs_d_ = (LocalSearchArgs *)(base + o_largs);
    sargs_d_ = (StatsArgs *)(base + o_sargs);
    uargs_d_ = (UpdateArgs *)(base + o_uargs);
    PrepArgs *pargs_d = (PrepArgs *)(base + o_pargs);
    items_d_ = (int2 *)(base + o_items);
    sw_items_d_ = (int2 *)(base + o_sw_items);
    ns_items_d_ = (int2 *)(base + o_ns_items);
    ls_needed_d_ = (uint8_t *)(base + o_ls_needed);
    route_desc_d_ = (int2 *)(base + o_rdesc);
    route_ctr_d_ = (int *)(base + o_rctr);
    route_rem_d_ = (int *)(base + o_rrem);
    ls_list_d_ = (int *)(base + o_lslist);
    ls_list_ctr_d_ = (int *)(base + o_lsctr);

    // ---- configuration (shared-memory budgets over the largest instance)
    const bool throughput = p.mode == ACO_MODE_THROUGHPUT;
    fin_any = false;
    long long max_routes = 1;
    int A_max = 1;
    for (const InstHost &ih : inst) {
        fin_any = fin_any || !std::isinf(ih.max_dist);
        long long dem = 0;
        for (int i = 1; i < ih.n; i++) dem += ih.demand[i];
        max_routes = std::max<long long>(max_routes, ih.capacity > 0 ? dem / ih.capacity + 1 : 1);
        A_max = std::max(A_max, ih.A);
    }
    if (!throughput) { // parity construct: warps per ant so that a thread owns <= 32 nodes of a row
        const InstHost &ih = inst[0];
        int wpa = 1;
        while (wpa < 8 && 32 * wpa * 32 < ih.n) wpa *= 2;
        while (wpa < 8 && ih.n > 256 * wpa && 32 * wpa * 2 <= ih.nloc) wpa *= 2;
        wpa = std::min(wpa, ih.nloc / 32);
        if (p.warps_per_ant > 0) wpa = p.warps_per_ant;
        cp_wpa = wpa;
        const int per_block = std::max(1, std::min(8, (ih.A + sm_count - 1) / sm_count));
        cp_apc = p.ants_per_block > 0 ? p.ants_per_block : std::max(1, per_block / wpa);
        if (cp_apc * cp_wpa > 16) return ACO_ERR_INVALID; // 512 threads per CTA at most
        cp_stage = construct_parity_smem(ih.n, ih.nloc, ih.kmax, wpa, cp_apc, true, fin_any) <= kSmemBudget;
    } else {
        // ants per work item: enough CTAs to cover the SMs for one instance,
        // larger items for big batches (the staging is shared by the item's ants)
        // (one warp per ant, at most 16 warps: the kernel's launch bound is 512 threads)
        if (p.ants_per_block > 0) cn_apc = std::min(16, p.ants_per_block);
        else if (count == 1) cn_apc = std::max(1, std::min(8, (inst[0].A + sm_count - 1) / sm_count));
        else cn_apc = std::max(1, std::min(16, total_ants / (sm_count * 2)));
        // helper draw warps while the construct is latency bound (few ants per SM)
        cn_draw = p.draw_warps > 0 || (p.draw_warps == 0 && p.construct_ctas != 2 && total_ants <= 4 * sm_count);
        if (cn_draw) cn_apc = std::min(cn_apc, 8);
        // two CTAs per SM (without helper draws or fused 2-opt) while there are
        // at least 32 ants an SM: the construct is latency bound per ant, and
        // twice the warps outweigh the tables that no longer fit in shared memory
        cn_wide = false;
        // shared-memory plan of every instance for `apc` ants per CTA and `lsw`
        // fused 2-opt warps (lsw > 0 needs the tables staged), within `budget` bytes a CTA
        auto plan = [&](int apc, int lsw, size_t budget) {
            const bool draw = cn_draw && lsw == 0 && apc <= 8;
            const bool wide = cn_wide && lsw == 0; // the two-CTA kernel stages no matrix, no table above 1024 nodes
            size_t mx = 0;
            for (InstHost &ih : inst) {
                bool packable = true;
                for (int i = 0; i < ih.n; i++)
                    if (ih.demand[i] < 0 || ih.demand[i] > 0xFFFF) packable = false;
                ih.smat = !wide && p.stage_matrix >= 0 && ih.n <= 1024 && packable &&
                          construct_nn_smem(ih.n, ih.K, ih.Kp, apc, true, true, false, lsw, draw) <= budget;
                ih.packed =
                    packable && construct_nn_smem(ih.n, ih.K, ih.Kp, apc, ih.smat, true, false, lsw, draw) <= budget;
                ih.gtab = false;
                size_t need = construct_nn_smem(ih.n, ih.K, ih.Kp, apc, ih.smat, ih.packed, false, lsw, draw);
                if (need > budget || (wide && ih.n > 1024)) {
                    ih.gtab = true; // the candidate table stays in global memory (read through L2)
                    ih.packed = packable;
                    need = construct_nn_smem(ih.n, ih.K, ih.Kp, apc, false, ih.packed, true, lsw, draw);
                }
                if (need > budget) return false;
                mx = std::max(mx, need);
            }
            cn_smem = mx;
            return true;
        };
        cn_lsw = 0;
        int n_max = 0;
        for (const InstHost &ih : inst) n_max = std::max(n_max, ih.n);
        if ((p.ls_flag & 1) && p.fuse_ls == 1 && n_max <= 1024) { // 2-opt fused into the construct
            // at most 4 constructing ants per CTA, the other warps (up to 16) improve
            // routes, so completed routes do not queue
            for (int apc = std::min(cn_apc, 4); apc >= 1 && cn_lsw == 0; apc--) {
                const int lsw = 16 - apc;
                if (plan(apc, lsw, kSmemBudget)) {
                    cn_apc = apc;
                    cn_lsw = lsw;
                }
            }
        }
        if (cn_lsw == 0) {
            cn_wide = !cn_draw && (p.construct_ctas == 2 || (p.construct_ctas == 0 && total_ants >= 32 * sm_count));
            const int apc0 = cn_apc;
            while (!plan(cn_apc, 0, cn_wide ? kWideBudget : kSmemBudget)) {
                if (cn_apc > 1) {
                    cn_apc--;
                } else if (cn_wide) { // not even one ant fits half an SM: one CTA per SM
                    cn_wide = false;
                    cn_apc = apc0;
                } else {
                    return ACO_ERR_INVALID; // candidate table of this size cannot be staged
                }
            }
        }
        cn_draw = cn_draw && cn_lsw == 0 && cn_apc <= 8; // as the last plan sized the shared memory
    }
    {
        // 2-opt CTA shape: ants per CTA x warps.  Cost model: waves of CTAs over
        // the SMs x (routes per warp + 1 for the CTA's set-up and write-back),
        // routes per ant estimated by total demand / capacity; ties go to more
        // warps per ant.  A caller's value is kept.
        int n_max = 0;
        for (const InstHost &ih : inst) n_max = std::max(n_max, ih.n);
        ls_nmax = n_max;
        long long best_cost = -1;
        double best_wpa = 0.0;
        ls_apc = 1;
        ls_warps = 1;
        ls_smem = local_search_smem(n_max, 1, 1);
        for (int apc = 1; apc <= 8; apc++) {
            if (p.ls_ants > 0 && apc != p.ls_ants) continue;
            int wcap = 32; // a caller's width is narrowed to what shared memory holds
            while (wcap > apc && local_search_smem(n_max, apc, wcap) > kSmemBudget) wcap--;
            for (int w = apc; w <= wcap; w++) {
                if (p.ls_warps > 0 && w != std::min(p.ls_warps, wcap)) continue;
                const size_t sm = local_search_smem(n_max, apc, w);
                if (sm > kSmemBudget) continue;
                const int res = local_search_occupancy(w, sm);
                if (res < 1) continue;
                const long long blocks = (total_ants + apc - 1) / apc;
                const long long waves = (blocks + (long long)res * sm_count - 1) / ((long long)res * sm_count);
                // + 1: the per-CTA set-up and write-back cost about one route
                const long long cost = waves * ((apc * max_routes + w - 1) / w + 1);
                const double wpa = (double)w / apc;
                if (best_cost < 0 || cost < best_cost || (cost == best_cost && wpa > best_wpa)) {
                    best_cost = cost;
                    best_wpa = wpa;
                    ls_apc = apc;
                    ls_warps = w;
                    ls_smem = sm;
                }
            }
        }
        if (best_cost < 0 && (p.ls_flag & 1)) return ACO_ERR_INVALID; // the caller's shape does not fit
    }
    if (p.ls_flag & 2) { // swap stage: as many ants per CTA as their shared arrays allow, up to 8
        int n_max = 0, ld_of_max = 32;
        for (const InstHost &ih : inst)
            if (ih.n > n_max) { n_max = ih.n; ld_of_max = ih.ld; }
        sw_apc = 8;
        while (sw_apc > 1 && swap_smem(n_max, ld_of_max, sw_apc) > kSmemBudget) sw_apc--;
        sw_smem = 0;
        for (const InstHost &ih : inst) sw_smem = std::max(sw_smem, swap_smem(ih.n, ih.ld, sw_apc));
        if (sw_smem > kSmemBudget) return ACO_ERR_INVALID; // the tour arrays of one ant do not fit
    }
    if (p.ns_rounds > 0) { // random-descent stage: up to 8 ants per CTA
        int n_max = 0;
        for (const InstHost &ih : inst) n_max = std::max(n_max, ih.n);
        ns_apc = 8;
        while (ns_apc > 1 && ns_smem(n_max, ns_apc) > kSmemBudget) ns_apc--;
        ns_smem_ = ns_smem(n_max, ns_apc);
        if (ns_smem_ > kSmemBudget) return ACO_ERR_INVALID;
    }
    stats_smem = (size_t)A_max * sizeof(float);
    if (stats_smem > kSmemBudget) return ACO_ERR_INVALID; // n_ants lengths must fit in shared memory

    // ---- host tables and uploads
    std::vector<int> ant_inst(total_ants), ant_base(count + 1), row_base(count + 1), row_inst(total_rows);
    std::vector<int2> items, swi, nsi;
    {
        int a0 = 0, r0 = 0;
        for (int b = 0; b < count; b++) {
            ant_base[b] = a0;
            row_base[b] = r0;
            for (int k = 0; k < inst[b].A; k++) ant_inst[a0 + k] = b;
            for (int k = 0; k < inst[b].n; k++) row_inst[r0 + k] = b;
            a0 += inst[b].A;
            r0 += inst[b].n;
        }
        ant_base[count] = a0;
        row_base[count] = r0;
        std::vector<int> order(count);
        for (int b = 0; b < count; b++) order[b] = b;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return inst[x].n > inst[y].n; });
        for (int b : order)
            for (int a0 = 0; a0 < inst[b].A; a0 += cn_apc) items.push_back(make_int2(b, a0));
        n_items = (int)items.size();
        for (int b = 0; b < count; b++)
            for (int a0 = 0; a0 < inst[b].A; a0 += sw_apc) swi.push_back(make_int2(b, a0));
        sw_items = (int)swi.size();
        for (int b = 0; b < count; b++)
            for (int a0 = 0; a0 < inst[b].A; a0 += ns_apc) nsi.push_back(make_int2(b, a0));
        ns_items = (int)nsi.size();
    }
    cargs_h_.resize(count);
    std::vector<LocalSearchArgs> largs(count);
    std::vector<StatsArgs> sargs(count);
    std::vector<UpdateArgs> uargs(count);
    const int ai = exp_as_int(p.alpha), bi = exp_as_int(p.beta);
    bool ok = true;
    // host -> device uploads are staged into one blob: one copy and one scatter
    // kernel per flush instead of a pageable copy per array
    Staging stage;
    auto up = [&](void *dst, const void *src, size_t bytes) { stage.add(dst, src, bytes); };
    for (int b = 0; b < count; b++) { // what the device preprocessing reads
        InstHost &ih = inst[b];
        std::vector<int> dem4(ih.n4, 0);
        std::copy(ih.demand.begin(), ih.demand.end(), dem4.begin());
        up(ih.dem_d, dem4.data(), dem4.size() * 4);
        if (ih.device_prep) {
            up(ih.xy_d, ih.x, (size_t)ih.n * 4);
            up(ih.xy_d + ih.n4, ih.y, (size_t)ih.n * 4);
        }
    }
    ok = ok && stage.flush(res->pool, sm_count, st) == cudaSuccess;
    std::vector<PrepArgs> pargs(count);
    int n_prep = 2; // the longest row the batched list kernel stages
    for (int b = 0; b < count; b++) {
        InstHost &ih = inst[b];
        const int n = ih.n;
        // distances, lists, tables (device_prep) and seeds: one launch each for the
        // whole batch after the uploads (prep.cu)
        PrepArgs &pa = pargs[b];
        pa = PrepArgs{};
        pa.n = n; pa.ld = ih.ld; pa.depth = ih.depth; pa.K = ih.K; pa.Kp = ih.Kp; pa.nn_ls = ih.nn_ls;
        pa.dist_type = ih.dist_type; pa.device_prep = ih.device_prep ? 1 : 0; pa.n_ants = ih.A;
        pa.x = ih.xy_d; pa.y = ih.xy_d ? ih.xy_d + ih.n4 : nullptr; pa.dist = ih.dist_d; pa.demand = ih.dem_d;
        pa.nn16 = ih.nn16_d; pa.cand32 = ih.cand32_d; pa.nnls = ih.nnls_d; pa.seeds = ih.seeds_d;
        if (ih.device_prep) {
            n_prep = std::max(n_prep, n);
        } else {
            ok = ok && cudaMemcpy2DAsync(ih.dist_d, (size_t)ih.ld * 4, ih.dist.data(), (size_t)n * 4, (size_t)n * 4,
                                         n, cudaMemcpyHostToDevice, st) == cudaSuccess;
        }
        if (!throughput) {
            const std::vector<int> prio = tournament_priority(n);
            std::vector<uint32_t> key(ih.n4, 0);
            for (int i = 0; i < n; i++) key[i] = ((uint32_t)(0xFFFF - prio[i]) << 16) | (uint32_t)i;
            std::vector<uint32_t> jump((ih.kmax + 3) & ~3, 0);
            for (int k = 0; k < ih.kmax; k++) jump[k] = pm_pow((uint64_t)k + 1);
            std::vector<uint32_t> adv(ih.nloc, 1);
            for (int l = 0; l < ih.nloc; l++)
                adv[l] = pm_pow(l < n ? (uint64_t)((n - l + ih.nloc - 1) / ih.nloc) : 0);
            up(ih.key_d, key.data(), key.size() * 4);
            up(ih.jump_d, jump.data(), jump.size() * 4);
            up(ih.adv_d, adv.data(), adv.size() * 4);
        }
        if (ih.K > 0 && !ih.device_prep) {
            std::vector<uint16_t> nn16((size_t)n * ih.Kp, 0);
            std::vector<uint32_t> cand32((size_t)n * ih.Kp, 0); // padding entries: node 0 (always visited)
            for (int i = 0; i < n; i++)
                for (int j = 0; j < ih.K; j++) {
                    const int c = ih.nn[(size_t)i * ih.depth + j];
                    nn16[(size_t)i * ih.Kp + j] = (uint16_t)c;
                    cand32[(size_t)i * ih.Kp + j] = (uint32_t)c | ((uint32_t)(ih.demand[c] & 0xFFFF) << 16);
                }
            up(ih.nn16_d, nn16.data(), nn16.size() * 2);
            up(ih.cand32_d, cand32.data(), cand32.size() * 4);
        }
        if (!ih.device_prep) {
            std::vector<int> nnls((size_t)n * std::max(1, ih.nn_ls), 0);
            for (int i = 0; i < n; i++)
                for (int j = 0; j < ih.nn_ls; j++) nnls[(size_t)i * ih.nn_ls + j] = ih.nn[(size_t)i * ih.depth + j];
            up(ih.nnls_d, nnls.data(), nnls.size() * 4);
        }

        ConstructArgs &c = cargs_h_[b];
        c = ConstructArgs{};
        c.n = n; c.ld = ih.ld; c.n_ants = ih.A; c.T = ih.T; c.nloc = ih.nloc; c.log2_nloc = ih.lg; c.kmax = ih.kmax;
        c.capacity = ih.capacity; c.max_dist = ih.max_dist; c.serv_time = ih.serv_time;
        c.total = ih.total_d; c.dist = ih.dist_d; c.demand = ih.dem_d; c.tiekey = ih.key_d; c.jump = ih.jump_d;
        c.adv = ih.adv_d; c.nn16 = ih.nn16_d; c.cand32 = ih.cand32_d; c.chc = ih.chc_d; c.K = ih.K; c.Kp = ih.Kp;
        c.smat = ih.smat ? 1 : 0; c.packed = ih.packed ? 1 : 0; c.gtab = ih.gtab ? 1 : 0;
        c.nn_list = ih.nnls_d; c.nn_ls = ih.nn_ls; c.pass_limit = p.ls_pass_limit; c.ant_base = ant_base[b];
        c.ls_best = p.ls_best;
        c.ls_needed = ls_needed_d_;
        c.route_desc = use_routes_ ? route_desc_d_ : nullptr;
        c.route_ctr = route_ctr_d_;
        c.route_rem = route_rem_d_;
        c.ls_list = ls_list_d_;
        c.ls_list_ctr = ls_list_ctr_d_;
        c.route_cap = route_cap_;
        c.seeds = ih.seeds_d; c.solutions = ih.sol_d; c.lens = ih.lens_d; c.status = status_d;
        c.wait_limit = wait_d;
        LocalSearchArgs &l = largs[b];
        l = LocalSearchArgs{};
        l.n = n; l.ld = ih.ld; l.n_ants = ih.A; l.T = ih.T; l.nn_ls = ih.nn_ls; l.rmax = 32;
        l.pass_limit = p.ls_pass_limit; l.dist = ih.dist_d; l.nn_list = ih.nnls_d; l.solutions = ih.sol_d;
        l.best = p.ls_best;
        l.lens = ih.lens_d; l.status = status_d;
        StatsArgs &s = sargs[b];
        s = StatsArgs{};
        s.n = n; s.n_ants = ih.A; s.T = ih.T; s.nloc = ih.nloc; s.log2_nloc = ih.lg; s.ras_ranks = ih.R;
        s.record_cap = p.record_cap; s.solutions = ih.sol_d; s.lens = ih.lens_d; s.elites = ih.elites_d;
        s.succ = ih.succ_d; s.depmask = ih.dep_d; s.d_tau = ih.dtau_d; s.num_bsf = ih.nbsf_d; s.records = ih.rec_d;
        s.iteration = ih.iter_d; s.t0_ns = t0_d_; s.status = status_d;
        UpdateArgs &u = uargs[b];
        u = UpdateArgs{};
        u.n = n; u.ld = ih.ld; u.ras_ranks = ih.R; u.evap = 1.0f - p.rho; u.alpha = p.alpha; u.beta = p.beta;
        u.alpha_int = ai; u.beta_int = bi; u.rho = p.rho; u.tau = ih.tau_d; u.total = ih.total_d; u.heur = ih.heur_d;
        u.dist = ih.dist_d; u.succ = ih.succ_d; u.depmask = ih.dep_d; u.d_tau = ih.dtau_d; u.bsf_len = ih.lens_d + ih.A;
        u.chc = ih.K > 0 ? ih.chc_d : nullptr; u.nn16 = ih.nn16_d; u.K = ih.K; u.Kp = ih.Kp;
    }
    up(cargs_d_, cargs_h_.data(), sizeof(ConstructArgs) * count);
    up(largs_d_, largs.data(), sizeof(LocalSearchArgs) * count);
    up(sargs_d_, sargs.data(), sizeof(StatsArgs) * count);
    stats_one_ = sargs[0];
    up(uargs_d_, uargs.data(), sizeof(UpdateArgs) * count);
    up(ant_inst_d_, ant_inst.data(), ant_inst.size() * 4);
    up(ant_base_d_, ant_base.data(), ant_base.size() * 4);
    up(row_base_d_, row_base.data(), row_base.size() * 4);
    up(row_inst_d_, row_inst.data(), row_inst.size() * 4);
    up(slot_base_d_, slot_base_h_.data(), slot_base_h_.size() * 4);
    up(tour_base_d_, tour_base_h_.data(), tour_base_h_.size() * 4);
    const int wl = std::max(0, p.wait_limit);
    up(wait_d, &wl, 4);
    up(items_d_, items.data(), items.size() * sizeof(int2));
    up(sw_items_d_, swi.data(), swi.size() * sizeof(int2));
    up(ns_items_d_, nsi.data(), nsi.size() * sizeof(int2));
    up(pargs_d, pargs.data(), sizeof(PrepArgs) * count);
    ok = ok && stage.flush(res->pool, sm_count, st) == cudaSuccess;
    if (!ok) return ACO_ERR_CUDA;
    CK(launch_prep_batch(pargs_d, row_base_d_, row_inst_d_, total_rows, n_prep, ant_base_d_, ant_inst_d_, total_ants,
                         p.nloc, p.seed_time, p.rnd_seed, status_d, sm_count, st));
    rc = run_rows(ROW_HEUR, 0.f);
    if (rc != ACO_OK) return rc;
    CK(cudaStreamSynchronize(st));
    for (InstHost &ih : inst) { // the host copies are no longer needed
        std::vector<int>().swap(ih.nn);
        std::vector<float>().swap(ih.dist);
        ih.x = ih.y = nullptr;
    }
    return sync_status();
}

int Colony::run_rows(int mode, float trail)
{
    CK(launch_rows(uargs_d_, row_base_d_, inst.size() > 1 ? row_inst_d_ : nullptr, total_rows, mode, trail, sm_count,
                   st));
    return ACO_OK;
}

int Colony::run_rows_one(int b, int mode)
{
    CK(launch_rows(uargs_d_ + b, zero_base_d_, nullptr, inst[b].n, mode, 0.f, sm_count, st));
    return ACO_OK;
}

int Colony::set_prior(int b, const float *prior, int ld)
{
    if (b < 0 || b >= (int)inst.size()) return ACO_ERR_INVALID;
    InstHost &ih = inst[b];
    const int n = ih.n;
    if (prior) {
        if (ld < n) return ACO_ERR_INVALID;
        for (int i = 0; i < n; i++) // weights must stay usable by the roulette
            for (int j = 0; j < n; j++) {
                const float v = prior[(size_t)i * ld + j];
                if (!(v >= 0.0f) || std::isinf(v)) return ACO_ERR_INVALID;
            }
    }
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    ih.prior_hash = 0;
    if (prior) {
        uint64_t hh = kFnvBasis;
        for (int i = 0; i < n; i++) hh = fnv1a(hh, prior + (size_t)i * ld, sizeof(float) * (size_t)n);
        ih.prior_hash = hh | 1u; // nonzero: a prior is set
        CK(cudaMemcpy2DAsync(ih.heur_d, (size_t)ih.ld * 4, prior, (size_t)ld * 4, (size_t)n * 4, n,
                             cudaMemcpyHostToDevice, st));
        rc = run_rows_one(b, ROW_PRIOR);
    } else {
        rc = run_rows_one(b, ROW_HEUR);
    }
    if (rc == ACO_OK && initialized) rc = run_rows_one(b, ROW_TOTAL);
    if (rc != ACO_OK) return rc;
    return sync_status();
}

int Colony::validate(int *flags, int *invalid_per_inst, int *n_invalid)
{
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    const int count = (int)inst.size();
    int a_max = 0, n_max = 0;
    for (const InstHost &ih : inst) {
        a_max = std::max(a_max, ih.A);
        n_max = std::max(n_max, ih.n);
    }
    CK(cudaMemsetAsync(invalid_d_, 0, sizeof(int) * count, st));
    CK(launch_validate(cargs_d_, count, a_max + 1, n_max, valid_d_, slot_base_d_, invalid_d_, st));
    std::vector<int> inv(count);
    CK(cudaMemcpyAsync(inv.data(), invalid_d_, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
    if (flags)
        CK(cudaMemcpyAsync(flags, valid_d_, sizeof(int) * slot_base_h_[count], cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    long long total = 0;
    for (int b = 0; b < count; b++) {
        total += inv[b];
        if (invalid_per_inst) invalid_per_inst[b] = inv[b];
    }
    if (n_invalid) *n_invalid = (int)total;
    return sync_status();
}

int Colony::get_best_all(int *tours, size_t cap_ints, int *sizes, float *lengths)
{
    const int count = (int)inst.size();
    if (tours && cap_ints < (size_t)tour_base_h_[count]) return ACO_ERR_CAPACITY;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    CK(launch_gather_best(cargs_d_, count, tour_base_d_, best_tours_d_, best_sizes_d_, best_lens_d_, st));
    if (tours) CK(cudaMemcpyAsync(tours, best_tours_d_, sizeof(int) * tour_base_h_[count], cudaMemcpyDeviceToHost, st));
    if (sizes) CK(cudaMemcpyAsync(sizes, best_sizes_d_, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
    if (lengths) CK(cudaMemcpyAsync(lengths, best_lens_d_, sizeof(float) * count, cudaMemcpyDeviceToHost, st));
    return sync_status();
}

// ---- checkpoint ---------------------------------------------------------
// File: the magic, a header describing the colony (count and the
// run-shaping parameters -- seed_time, rnd_seed, ls_flag, ns_rounds,
// record_cap, mode -- then per instance n, A, nloc, K, nn_ls, ras_ranks, the
// fp32 bits of alpha, beta, rho, and the 64-bit hashes of the instance's data
// and of its prior), then per instance its iteration counter, number of
// best-so-far records, tau (n x n), tours and lengths (the reference layout),
// lane seeds and records.  Integers and floats are stored in host byte order.
namespace {
constexpr char kMagic[8] = {'A', 'C', 'O', 'C', 'K', 'P', 'T', '2'};

struct FileCloser {
    FILE *f;
    ~FileCloser()
    {
        if (f) std::fclose(f);
    }
};
} // namespace

static std::vector<int> checkpoint_header(const Colony &c)
{
    std::vector<int> h;
    const int run[] = {(int)c.inst.size(), c.p.seed_time, c.p.rnd_seed, c.p.ls_flag, c.p.ns_rounds, c.p.record_cap,
                       c.p.mode};
    h.insert(h.end(), run, run + sizeof(run) / sizeof(run[0]));
    for (const InstHost &ih : c.inst) {
        int a, b, r;
        std::memcpy(&a, &c.p.alpha, 4);
        std::memcpy(&b, &c.p.beta, 4);
        std::memcpy(&r, &c.p.rho, 4);
        const int v[] = {ih.n, ih.A, ih.nloc, ih.K, ih.nn_ls, ih.R, a, b, r,
                         (int)(uint32_t)ih.data_hash, (int)(uint32_t)(ih.data_hash >> 32),
                         (int)(uint32_t)ih.prior_hash, (int)(uint32_t)(ih.prior_hash >> 32)};
        h.insert(h.end(), v, v + sizeof(v) / sizeof(v[0]));
    }
    return h;
}

int Colony::save_checkpoint(const char *path)
{
    if (!path) return ACO_ERR_INVALID;
    if (!initialized) return ACO_ERR_STATE;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    rc = sync_status();
    if (rc != ACO_OK) return rc;
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return ACO_ERR_IO;
    const std::vector<int> h = checkpoint_header(*this);
    const int hn = (int)h.size();
    bool ok = std::fwrite(kMagic, 1, 8, fc.f) == 8 && std::fwrite(&hn, 4, 1, fc.f) == 1 &&
              std::fwrite(h.data(), 4, h.size(), fc.f) == h.size();
    for (const InstHost &ih : inst) {
        if (!ok) break;
        const size_t nn = (size_t)ih.n * ih.n, ns = (size_t)ih.T * (ih.A + 1) + 1, nseed = (size_t)ih.A * ih.nloc;
        int it = 0, nb = 0;
        std::vector<float> tau(nn), lens(ih.A + 1);
        std::vector<int> sol(ns), seeds(nseed);
        std::vector<aco_record> rec(p.record_cap);
        CK(cudaMemcpyAsync(&it, ih.iter_d, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&nb, ih.nbsf_d, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpy2DAsync(tau.data(), (size_t)ih.n * 4, ih.tau_d, (size_t)ih.ld * 4, (size_t)ih.n * 4, ih.n,
                             cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(sol.data(), ih.sol_d, ns * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(lens.data(), ih.lens_d, lens.size() * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(seeds.data(), ih.seeds_d, nseed * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rec.data(), ih.rec_d, rec.size() * sizeof(aco_record), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ok = std::fwrite(&it, 4, 1, fc.f) == 1 && std::fwrite(&nb, 4, 1, fc.f) == 1 &&
             std::fwrite(tau.data(), 4, nn, fc.f) == nn && std::fwrite(sol.data(), 4, ns, fc.f) == ns &&
             std::fwrite(lens.data(), 4, lens.size(), fc.f) == lens.size() &&
             std::fwrite(seeds.data(), 4, nseed, fc.f) == nseed &&
             std::fwrite(rec.data(), sizeof(aco_record), rec.size(), fc.f) == rec.size();
    }
    if (!ok) return ACO_ERR_IO;
    const int cr = std::fclose(fc.f);
    fc.f = nullptr;
    return cr == 0 ? ACO_OK : ACO_ERR_IO;
}

int Colony::load_checkpoint(const char *path)
{
    if (!path) return ACO_ERR_INVALID;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return ACO_ERR_IO;
    char magic[8];
    int hn = 0;
    if (std::fread(magic, 1, 8, fc.f) != 8 || std::memcmp(magic, kMagic, 8) != 0) return ACO_ERR_IO;
    const std::vector<int> want = checkpoint_header(*this);
    if (std::fread(&hn, 4, 1, fc.f) != 1 || hn != (int)want.size()) return ACO_ERR_INVALID;
    std::vector<int> h(hn);
    if (std::fread(h.data(), 4, h.size(), fc.f) != h.size()) return ACO_ERR_IO;
    if (h != want) return ACO_ERR_INVALID; // another instance set or other parameters
    for (InstHost &ih : inst) {
        const size_t nn = (size_t)ih.n * ih.n, ns = (size_t)ih.T * (ih.A + 1) + 1, nseed = (size_t)ih.A * ih.nloc;
        int it = 0, nb = 0;
        std::vector<float> tau(nn), lens(ih.A + 1);
        std::vector<int> sol(ns), seeds(nseed);
        std::vector<aco_record> rec(p.record_cap);
        const bool ok = std::fread(&it, 4, 1, fc.f) == 1 && std::fread(&nb, 4, 1, fc.f) == 1 &&
                        std::fread(tau.data(), 4, nn, fc.f) == nn && std::fread(sol.data(), 4, ns, fc.f) == ns &&
                        std::fread(lens.data(), 4, lens.size(), fc.f) == lens.size() &&
                        std::fread(seeds.data(), 4, nseed, fc.f) == nseed &&
                        std::fread(rec.data(), sizeof(aco_record), rec.size(), fc.f) == rec.size();
        if (!ok) return ACO_ERR_IO;
        CK(cudaMemcpyAsync(ih.iter_d, &it, 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ih.nbsf_d, &nb, 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpy2DAsync(ih.tau_d, (size_t)ih.ld * 4, tau.data(), (size_t)ih.n * 4, (size_t)ih.n * 4, ih.n,
                             cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ih.sol_d, sol.data(), ns * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ih.lens_d, lens.data(), lens.size() * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ih.seeds_d, seeds.data(), nseed * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ih.rec_d, rec.data(), rec.size() * sizeof(aco_record), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st)); // the host vectors go out of scope
    }
    rc = run_rows(ROW_TOTAL, 0.f); // total_info and the candidate table from the restored tau
    if (rc != ACO_OK) return rc;
    CK(cudaMemsetAsync(status_d, 0, sizeof(int), st));
    CK(launch_t0(t0_d_, st)); // record times restart from the resume
    t_init = std::chrono::steady_clock::now();
    rc = sync_status();
    if (rc == ACO_OK) initialized = true;
    return rc;
}

int Colony::construct(bool in_iteration)
{
    const bool fused = in_iteration;
    if (p.mode != ACO_MODE_THROUGHPUT) {
        CK(launch_construct_parity(cargs_h_[0], cp_wpa, cp_apc, cp_stage, st));
        return ACO_OK;
    }
    const int lsw = fused && p.ls_flag ? cn_lsw : 0; // the queue starts at 0 (zeroed arena, rewound by the kernel)
    last_fused_ = lsw > 0;
    // the route list is rewound by the 2-opt kernel that consumes it; a second
    // construct without one in between starts it afresh
    if (use_routes_ && lsw == 0 && routes_pending_) {
        CK(cudaMemsetAsync(route_ctr_d_, 0, 16, st));
        CK(cudaMemsetAsync(ls_list_ctr_d_, 0, 16, st));
    }
    routes_pending_ = use_routes_ && lsw == 0;
    // inside an iteration the 2-opt follows and, with the route list, writes every tour length
    const bool lens_later = in_iteration && routes_pending_ && (p.ls_flag & 1);
    CK(launch_construct_nn(cargs_d_, items_d_, n_items, queue_d_, cn_apc, cn_smem, sm_count, fin_any, st, lsw,
                           cn_draw, lens_later, cn_wide && lsw == 0));
    return ACO_OK;
}

int Colony::local_search()
{
    // after a fused construct or the route-level kernel, only the ants marked
    // in ls_needed still need the per-ant kernel
    const bool routes = routes_pending_;
    if (routes)
        CK(launch_route_opt(largs_d_, ant_inst_d_, ant_base_d_, route_desc_d_, route_ctr_d_, route_cap_, route_rem_d_,
                            ls_needed_d_, ls_nmax, kRouteWarps, sm_count, st));
    routes_pending_ = false;
    // after the route-level kernel only the ants the construct listed remain: a
    // persistent grid over that list; after a fused construct, every ant's flag
    CK(launch_local_search(largs_d_, ant_inst_d_, ant_base_d_, total_ants, ls_apc, ls_nmax, ls_warps, ls_smem, st,
                           last_fused_ || routes ? ls_needed_d_ : nullptr, routes ? ls_list_d_ : nullptr,
                           routes ? ls_list_ctr_d_ : nullptr, sm_count));
    last_fused_ = false;
    if (p.ls_flag & 2) CK(launch_swap(cargs_d_, sw_items_d_, sw_items, sw_apc, sw_smem, kSwapLimitPerNode, st));
    return ACO_OK;
}

int Colony::neighbourhood()
{
    CK(launch_ns(cargs_d_, sargs_d_, ns_items_d_, ns_items, ns_apc, ns_smem_, p.ns_rounds, p.rnd_seed, st));
    return ACO_OK;
}

int Colony::stats(bool elites)
{
    CK(launch_stats(sargs_d_, (int)inst.size(), elites ? 1 : 0, stats_smem, st, inst.size() == 1 ? &stats_one_ : nullptr));
    return ACO_OK;
}

int Colony::update() { return run_rows(ROW_UPDATE, 0.f); }

int Colony::pheromone_init(float trail, bool from_bsf)
{
    return run_rows(from_bsf ? ROW_INIT_BSF : ROW_INIT_TRAIL, trail);
}

int Colony::gather_candidates() { return p.mode == ACO_MODE_THROUGHPUT ? run_rows(ROW_GATHER, 0.f) : ACO_OK; }

int Colony::run_phases()
{
    int rc = construct(true);
    if (rc == ACO_OK && p.ls_flag) rc = local_search();
    if (rc == ACO_OK && p.ns_rounds > 0) rc = neighbourhood();
    if (rc == ACO_OK) rc = stats(true);
    if (rc == ACO_OK) rc = update();
    return rc;
}

int Colony::launches_per_iteration() const
{
    int k = 3; // construct, statistics, pheromone pass
    if (p.ls_flag) k += 1 + (use_routes_ && cn_lsw == 0 ? 1 : 0) + ((p.ls_flag & 2) ? 1 : 0); // 2-opt kernels, swap
    if (p.ns_rounds > 0) k += 1;
    return k;
}

int Colony::set_wait_limit(int polls)
{
    if (polls < 0) return ACO_ERR_INVALID;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    h_pin[3] = polls; // pinned: the copy is ordered on the stream, the word read by the next launch
    CK(cudaMemcpyAsync(wait_d, h_pin + 3, sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    p.wait_limit = polls;
    return ACO_OK;
}

int Colony::clear_status()
{
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    const int prev = sync_status();
    CK(cudaMemsetAsync(status_d, 0, sizeof(int), st));
    CK(cudaStreamSynchronize(st));
    return prev;
}

int Colony::sync_status()
{
    CK(cudaMemcpyAsync(h_pin, status_d, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return h_pin[0];
}

int Colony::ensure_graph()
{
    if (exec_) return ACO_OK;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = run_phases();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != ACO_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc != ACO_OK ? rc : ACO_ERR_CUDA;
    }
    graph_ = g;
    CK(cudaGraphInstantiate(&exec_, g, 0));
    return ACO_OK;
}

int Colony::init()
{
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    CK(launch_reset_slots(sargs_d_, (int)inst.size(), st));
    CK(cudaMemsetAsync(status_d, 0, sizeof(int), st));
    CK(launch_t0(t0_d_, st));
    t_init = std::chrono::steady_clock::now();
    // g_aco.cpp:79-92
    rc = pheromone_init(0.5f, false);
    if (rc == ACO_OK) rc = construct(true);
    if (rc == ACO_OK && p.ls_flag) rc = local_search();
    if (rc == ACO_OK) rc = stats(false);
    if (rc == ACO_OK) rc = pheromone_init(0.f, true);
    if (rc != ACO_OK) return rc;
    // the iteration graph is captured and instantiated on the host while the
    // device runs the initial iteration (capture records, it does not run)
    if (p.use_graph) rc = ensure_graph();
    const int status = sync_status();
    initialized = status == ACO_OK && rc == ACO_OK;
    return status != ACO_OK ? status : rc;
}

int Colony::enqueue(int n_iter)
{
    if (!initialized) return ACO_ERR_STATE;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    if (p.use_graph) {
        rc = ensure_graph();
        if (rc != ACO_OK) return rc;
        for (int i = 0; i < n_iter; i++) CK(cudaGraphLaunch(exec_, st));
        return ACO_OK;
    }
    for (int i = 0; i < n_iter && rc == ACO_OK; i++) rc = run_phases();
    return rc;
}

int Colony::time_phases(int n_iter, float *ms4)
{
    if (!initialized) return ACO_ERR_STATE;
    int rc = set_device();
    if (rc != ACO_OK) return rc;
    cudaEvent_t ev[5];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    for (int k = 0; k < 4; k++) ms4[k] = 0.f;
    for (int it = 0; it < n_iter && rc == ACO_OK; it++) {
        CK(cudaEventRecord(ev[0], st));
        rc = construct(true);
        CK(cudaEventRecord(ev[1], st));
        if (rc == ACO_OK && p.ls_flag) rc = local_search();
        if (rc == ACO_OK && p.ns_rounds > 0) rc = neighbourhood();
        CK(cudaEventRecord(ev[2], st));
        if (rc == ACO_OK) rc = stats(true);
        CK(cudaEventRecord(ev[3], st));
        if (rc == ACO_OK) rc = update();
        CK(cudaEventRecord(ev[4], st));
        CK(cudaEventSynchronize(ev[4]));
        for (int k = 0; k < 4; k++) {
            float m = 0.f;
            CK(cudaEventElapsedTime(&m, ev[k], ev[k + 1]));
            ms4[k] += m;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc != ACO_OK) return rc;
    return sync_status();
}

} // namespace aco
