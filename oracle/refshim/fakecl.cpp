/*
 * fakecl.cpp -- a CPU stand-in for the OpenCL runtime, so that the reference's
 * unmodified host code (cvrp_ocl/gpu/g_type.cpp, g_aco.cpp) and kernels
 * (cvrp_ocl/gpu/kernel.cl, compiled as C++ with kernel_shim.h) run here.
 * TEST INFRASTRUCTURE ONLY: it pins the oracle restatement to the reference.
 *
 * Buffers are host allocations.  clEnqueueNDRangeKernel runs every work-group
 * one after another.  Kernels that call barrier() run their work-items as
 * cooperative coroutines (a hand-rolled x86-64 stack switch), so each barrier is
 * a real rendezvous of the whole work-group, exactly as on a device.  Kernels
 * without barriers run their work-items in order on the caller's stack.
 * time() is interposed so the reference's time-based seeds are reproducible.
 */
#include "CL/cl.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

/* ---- values the driver sets ------------------------------------------- */
extern "C" {
int fcl_num_node = 0;
int fcl_n_ants = 0;
int fcl_max_wg = 1024;
long fcl_fake_time = 0;
}

/* time(NULL) replacement (g_aco.cpp:718, problem.cpp:212). The library is linked
 * with -Bsymbolic-functions so the reference objects bind to this definition. */
extern "C" time_t time(time_t *t)
{
    if (t) *t = (time_t)fcl_fake_time;
    return (time_t)fcl_fake_time;
}

void display_ocl_info(void) {} /* OpenCLInfo.h; gated off by display_ocl_flag */

struct _cl_mem {
    size_t size;
    char *data;
};
struct _cl_platform_id { int dummy; };
struct _cl_device_id { int dummy; };
struct _cl_context { int dummy; };
struct _cl_command_queue { int dummy; };
struct _cl_program { int dummy; };
struct _cl_event { int dummy; };

struct KArg {
    bool set = false, is_local = false;
    size_t size = 0;
    std::vector<char> value;
};
struct _cl_kernel {
    std::string name;
    KArg args[32];
};

static _cl_platform_id g_platform;
static _cl_device_id g_device;
static _cl_context g_context;
static _cl_command_queue g_queue;
static _cl_program g_program;
static _cl_event g_event;

extern "C" void *fcl_mem_data(cl_mem m) { return m ? m->data : nullptr; }
extern "C" size_t fcl_mem_size(cl_mem m) { return m ? m->size : 0; }

/* ---- work-item state and the coroutine switch ------------------------- */
struct WorkItem {
    size_t gid, lid, grp;
    void *sp;
    bool done;
    int barriers;
};
static WorkItem *g_cur = nullptr;
static size_t g_local_size = 1;
static bool g_coroutine_mode = false;
static void *g_sched_sp = nullptr;
static void (*g_body)(cl_kernel) = nullptr;
static cl_kernel g_body_kernel = nullptr;
static std::vector<char *> g_stacks;
static const size_t kStack = 256 * 1024;

extern "C" void fcl_switch(void **save_sp, void *load_sp);
__asm__(".text\n"
        ".globl fcl_switch\n"
        ".hidden fcl_switch\n"
        ".type fcl_switch, @function\n"
        "fcl_switch:\n"
        "  pushq %rbp\n  pushq %rbx\n  pushq %r12\n  pushq %r13\n  pushq %r14\n  pushq %r15\n"
        "  movq %rsp, (%rdi)\n"
        "  movq %rsi, %rsp\n"
        "  popq %r15\n  popq %r14\n  popq %r13\n  popq %r12\n  popq %rbx\n  popq %rbp\n"
        "  ret\n"
        ".size fcl_switch, .-fcl_switch\n");

static void wi_entry()
{
    g_body(g_body_kernel);
    g_cur->done = true;
    fcl_switch(&g_cur->sp, g_sched_sp);
    abort(); /* never resumed */
}

size_t fcl_get_global_id(unsigned) { return g_cur->gid; }
size_t fcl_get_local_id(unsigned) { return g_cur->lid; }
size_t fcl_get_group_id(unsigned) { return g_cur->grp; }
size_t fcl_get_local_size(unsigned) { return g_local_size; }

void fcl_barrier(void)
{
    if (!g_coroutine_mode) {
        fprintf(stderr, "fakecl: barrier() in a kernel run without work-group emulation\n");
        abort();
    }
    g_cur->barriers++;
    fcl_switch(&g_cur->sp, g_sched_sp);
}

unsigned fcl_atomic_cmpxchg(volatile unsigned *p, unsigned cmp, unsigned val)
{
    unsigned old = *p;
    if (old == cmp) *p = val;
    return old;
}

float fcl_pow(float x, float e)
{
    if (e == 1.0f) return x;
    if (e >= 0.0f && e <= 8.0f && e == (float)(int)e) {
        int k = (int)e;
        if (k == 0) return 1.0f;
        float r = x;
        for (int i = 1; i < k; i++) r = r * x;
        return r;
    }
    return powf(x, e);
}

/* ---- argument access for the kernel wrappers ------------------------- */
static std::vector<std::vector<char>> g_local_bufs;

template <class T> static T scal(cl_kernel k, int i)
{
    T v;
    memcpy(&v, k->args[i].value.data(), sizeof(T));
    return v;
}
template <class T> static T *buf(cl_kernel k, int i)
{
    if (k->args[i].is_local) return reinterpret_cast<T *>(g_local_bufs[i].data());
    cl_mem m = scal<cl_mem>(k, i);
    return m ? reinterpret_cast<T *>(m->data) : nullptr;
}

/* the reference kernels, compiled from kernel.cl inside namespace oclk */
namespace oclk {
struct BestSolutionInfo;
void construct_solution(const int, const float, const float, int *, float *, int *, float *, int *,
                        float *, float *, int *, float *, float *, bool *, bool *, float *, int *);
void local_search(const int, int *, float *, int *, float *, int *, const int, const float, const float);
void update_best_so_far(bool *, int *, float *, BestSolutionInfo *, int *, float, int);
void best_solution_phase_0(int, float *, float *, int *, float *, int *);
void best_solution_phase_1(int, int *, float *, float *, int *, bool *);
void pheromone_init(float, float *, float *, float *);
void pheromone_evaporation(float *);
void update_pheromone_weighted(float *, int *, int, float, int);
void get_elites(float *, int *);
void pheromone_deposit(int *, int *, float *, float *, int *);
void compute_total_info(float *, float *, float *);
void update_best_so_far_to_device(int *, int, float, int *, float *);
} // namespace oclk

static void k_construct(cl_kernel k)
{
    oclk::construct_solution(scal<int>(k, 0), scal<float>(k, 1), scal<float>(k, 2), buf<int>(k, 3),
                             buf<float>(k, 4), buf<int>(k, 5), buf<float>(k, 6), buf<int>(k, 7),
                             buf<float>(k, 8), buf<float>(k, 9), buf<int>(k, 10), buf<float>(k, 11),
                             buf<float>(k, 12), buf<bool>(k, 13), buf<bool>(k, 14), buf<float>(k, 15),
                             buf<int>(k, 16));
}
static void k_local_search(cl_kernel k)
{
    oclk::local_search(scal<int>(k, 0), buf<int>(k, 1), buf<float>(k, 2), buf<int>(k, 3), buf<float>(k, 4),
                       buf<int>(k, 5), scal<int>(k, 6), scal<float>(k, 7), scal<float>(k, 8));
}
static void k_update_bsf(cl_kernel k)
{
    oclk::update_best_so_far(buf<bool>(k, 0), buf<int>(k, 1), buf<float>(k, 2),
                             buf<oclk::BestSolutionInfo>(k, 3), buf<int>(k, 4), scal<float>(k, 5),
                             scal<int>(k, 6));
}
static void k_best0(cl_kernel k)
{
    oclk::best_solution_phase_0(scal<int>(k, 0), buf<float>(k, 1), buf<float>(k, 2), buf<int>(k, 3),
                                buf<float>(k, 4), buf<int>(k, 5));
}
static void k_best1(cl_kernel k)
{
    oclk::best_solution_phase_1(scal<int>(k, 0), buf<int>(k, 1), buf<float>(k, 2), buf<float>(k, 3),
                                buf<int>(k, 4), buf<bool>(k, 5));
}
static void k_ph_init(cl_kernel k)
{
    oclk::pheromone_init(scal<float>(k, 0), buf<float>(k, 1), buf<float>(k, 2), buf<float>(k, 3));
}
static void k_evap(cl_kernel k) { oclk::pheromone_evaporation(buf<float>(k, 0)); }
static void k_weighted(cl_kernel k)
{
    oclk::update_pheromone_weighted(buf<float>(k, 0), buf<int>(k, 1), scal<int>(k, 2), scal<float>(k, 3),
                                    scal<int>(k, 4));
}
static void k_elites(cl_kernel k) { oclk::get_elites(buf<float>(k, 0), buf<int>(k, 1)); }
static void k_deposit(cl_kernel k)
{
    oclk::pheromone_deposit(buf<int>(k, 0), buf<int>(k, 1), buf<float>(k, 2), buf<float>(k, 3), buf<int>(k, 4));
}
static void k_total(cl_kernel k) { oclk::compute_total_info(buf<float>(k, 0), buf<float>(k, 1), buf<float>(k, 2)); }
static void k_to_device(cl_kernel k)
{
    oclk::update_best_so_far_to_device(buf<int>(k, 0), scal<int>(k, 1), scal<float>(k, 2), buf<int>(k, 3),
                                       buf<float>(k, 4));
}

struct KDesc {
    const char *name;
    void (*fn)(cl_kernel);
    bool uses_barrier;
};
static const KDesc kKernels[] = {
    {"construct_solution", k_construct, true},
    {"local_search", k_local_search, false},
    {"pheromone_init", k_ph_init, false},
    {"pheromone_evaporation", k_evap, false},
    {"pheromone_deposit", k_deposit, true},
    {"update_pheromone_weighted", k_weighted, false},
    {"compute_total_info", k_total, false},
    {"get_elites", k_elites, false},
    {"update_best_so_far", k_update_bsf, false},
    {"update_best_so_far_to_device", k_to_device, false},
    {"best_solution_phase_0", k_best0, true},
    {"best_solution_phase_1", k_best1, false},
};

static const KDesc *find_kernel(const std::string &name)
{
    for (const KDesc &d : kKernels)
        if (name == d.name) return &d;
    return nullptr;
}

/* ---- the API ---------------------------------------------------------- */
extern "C" {

cl_int clGetPlatformIDs(cl_uint, cl_platform_id *p, cl_uint *n)
{
    if (p) *p = &g_platform;
    if (n) *n = 1;
    return CL_SUCCESS;
}

cl_context clCreateContextFromType(const cl_context_properties *, cl_device_type,
                                   void (*)(const char *, const void *, size_t, void *), void *, cl_int *e)
{
    if (e) *e = CL_SUCCESS;
    return &g_context;
}

cl_int clGetContextInfo(cl_context, cl_context_info info, size_t size, void *value, size_t *ret)
{
    if (info != CL_CONTEXT_DEVICES) return CL_INVALID_VALUE;
    if (ret) *ret = sizeof(cl_device_id);
    if (value && size >= sizeof(cl_device_id)) *(cl_device_id *)value = &g_device;
    return CL_SUCCESS;
}

cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_command_queue_properties, cl_int *e)
{
    if (e) *e = CL_SUCCESS;
    return &g_queue;
}

cl_program clCreateProgramWithSource(cl_context, cl_uint count, const char **src, const size_t *, cl_int *e)
{
    /* g_type.cpp:193-200 prepends "#define NUM_NODE n\n#define N_ANTS a\n" */
    for (cl_uint i = 0; i < count; i++) {
        const char *p = strstr(src[i], "#define NUM_NODE ");
        if (p) fcl_num_node = atoi(p + strlen("#define NUM_NODE "));
        p = strstr(src[i], "#define N_ANTS ");
        if (p) fcl_n_ants = atoi(p + strlen("#define N_ANTS "));
    }
    if (e) *e = CL_SUCCESS;
    return &g_program;
}

cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id *, const char *, void (*)(cl_program, void *), void *)
{
    return CL_SUCCESS;
}

cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t size, void *value, size_t *ret)
{
    if (ret) *ret = 1;
    if (value && size >= 1) ((char *)value)[0] = 0;
    return CL_SUCCESS;
}

cl_int clGetDeviceInfo(cl_device_id, cl_device_info info, size_t, void *value, size_t *ret)
{
    /* the caller passes sizeof(size_t) for an int member (g_type.cpp:71-72);
     * only an int is written here */
    int v = 0;
    if (info == CL_DEVICE_MAX_WORK_GROUP_SIZE) v = fcl_max_wg;
    else if (info == CL_DEVICE_MAX_COMPUTE_UNITS) v = 1;
    if (value) memcpy(value, &v, sizeof(int));
    if (ret) *ret = sizeof(int);
    return CL_SUCCESS;
}

cl_kernel clCreateKernel(cl_program, const char *name, cl_int *e)
{
    if (!find_kernel(name)) {
        if (e) *e = CL_INVALID_KERNEL_NAME;
        return nullptr;
    }
    cl_kernel k = new _cl_kernel;
    k->name = name;
    if (e) *e = CL_SUCCESS;
    return k;
}

cl_int clReleaseCommandQueue(cl_command_queue) { return CL_SUCCESS; }
cl_int clReleaseKernel(cl_kernel k) { delete k; return CL_SUCCESS; }
cl_int clReleaseProgram(cl_program) { return CL_SUCCESS; }
cl_int clReleaseContext(cl_context) { return CL_SUCCESS; }
cl_int clReleaseDevice(cl_device_id) { return CL_SUCCESS; }

cl_int clReleaseMemObject(cl_mem m)
{
    if (m) { free(m->data); delete m; }
    return CL_SUCCESS;
}

cl_mem clCreateBuffer(cl_context, cl_mem_flags flags, size_t size, void *host, cl_int *e)
{
    cl_mem m = new _cl_mem;
    m->size = size;
    m->data = (char *)calloc(size ? size : 1, 1);
    if ((flags & CL_MEM_COPY_HOST_PTR) && host) memcpy(m->data, host, size);
    if (e) *e = CL_SUCCESS;
    return m;
}

cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem m, cl_bool, size_t off, size_t size, const void *src,
                            cl_uint, const cl_event *, cl_event *ev)
{
    if (off + size > m->size) return CL_INVALID_VALUE;
    memcpy(m->data + off, src, size);
    if (ev) *ev = &g_event;
    return CL_SUCCESS;
}

cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem m, cl_bool, size_t off, size_t size, void *dst,
                           cl_uint, const cl_event *, cl_event *ev)
{
    if (off + size > m->size) return CL_INVALID_VALUE;
    memcpy(dst, m->data + off, size);
    if (ev) *ev = &g_event;
    return CL_SUCCESS;
}

cl_int clSetKernelArg(cl_kernel k, cl_uint idx, size_t size, const void *value)
{
    if (idx >= 32) return CL_INVALID_VALUE;
    KArg &a = k->args[idx];
    a.set = true;
    a.size = size;
    a.is_local = (value == nullptr);
    a.value.assign(size, 0);
    if (value) memcpy(a.value.data(), value, size);
    return CL_SUCCESS;
}

cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel k, cl_uint, const size_t *, const size_t *gws,
                              const size_t *lws, cl_uint, const cl_event *, cl_event *ev)
{
    const KDesc *d = find_kernel(k->name);
    size_t global = gws[0];
    size_t local = lws ? lws[0] : 1;
    if (local == 0 || global % local != 0) return CL_INVALID_VALUE;
    size_t groups = global / local;
    g_local_size = local;
    g_body = d->fn;
    g_body_kernel = k;
    g_local_bufs.assign(32, std::vector<char>());
    if (d->uses_barrier)
        while (g_stacks.size() < local) g_stacks.push_back((char *)malloc(kStack));
    std::vector<WorkItem> items(local);
    for (size_t grp = 0; grp < groups; grp++) {
        for (int i = 0; i < 32; i++) /* __local arguments: fresh per work-group */
            if (k->args[i].set && k->args[i].is_local) g_local_bufs[i].assign(k->args[i].size + 64, 0);
        for (size_t lid = 0; lid < local; lid++) {
            WorkItem &w = items[lid];
            w.gid = grp * local + lid;
            w.lid = lid;
            w.grp = grp;
            w.done = false;
            w.barriers = 0;
        }
        if (!d->uses_barrier) {
            g_coroutine_mode = false;
            for (size_t lid = 0; lid < local; lid++) {
                g_cur = &items[lid];
                g_body(k);
            }
            continue;
        }
        g_coroutine_mode = true;
        for (size_t lid = 0; lid < local; lid++) {
            char *top = g_stacks[lid] + kStack;
            top = (char *)((uintptr_t)top & ~(uintptr_t)15);
            void **sp = (void **)top;
            *--sp = nullptr;           /* fake return address of wi_entry */
            *--sp = (void *)&wi_entry; /* popped by ret */
            for (int r = 0; r < 6; r++) *--sp = nullptr; /* r15 r14 r13 r12 rbx rbp */
            items[lid].sp = sp;
        }
        size_t alive = local;
        while (alive > 0) {
            for (size_t lid = 0; lid < local; lid++) {
                if (items[lid].done) continue;
                g_cur = &items[lid];
                fcl_switch(&g_sched_sp, items[lid].sp);
            }
            alive = 0;
            int bar = -1;
            for (size_t lid = 0; lid < local; lid++) {
                if (items[lid].done) continue;
                alive++;
                if (bar < 0) bar = items[lid].barriers;
                else if (bar != items[lid].barriers) {
                    fprintf(stderr, "fakecl: divergent barrier in %s\n", k->name.c_str());
                    abort();
                }
            }
            if (alive > 0 && alive != local) {
                fprintf(stderr, "fakecl: work-items of %s left the kernel at different barriers\n", k->name.c_str());
                abort();
            }
        }
        g_coroutine_mode = false;
    }
    if (ev) *ev = &g_event;
    return CL_SUCCESS;
}

cl_int clFinish(cl_command_queue) { return CL_SUCCESS; }
cl_int clWaitForEvents(cl_uint, const cl_event *) { return CL_SUCCESS; }

cl_int clGetEventProfilingInfo(cl_event, cl_profiling_info, size_t size, void *value, size_t *ret)
{
    if (value && size >= sizeof(cl_ulong)) *(cl_ulong *)value = 0;
    if (ret) *ret = sizeof(cl_ulong);
    return CL_SUCCESS;
}

} /* extern "C" */
