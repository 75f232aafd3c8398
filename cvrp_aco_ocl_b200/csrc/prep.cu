// prep.cu -- instance preprocessing on the device: the distance matrix
// (compute_distances, vrpHelper.cpp:160-184, with the per-type formulas of
// vrpHelper.cpp:35-158) and the nearest-neighbour lists (compute_nn_lists,
// vrpHelper.cpp:188-236, sorted by utilities.cpp:246-266), bit-identical to
// the host versions in host.cpp.
//
// Distances: EUC_2D, CEIL_2D and ATT use only correctly rounded operations
// (fp32 products and sums, fp32 or fp64 square root and division), so the
// device reproduces the host bits.  GEO goes through cos/acos, whose last bits
// differ between math libraries; it stays on the host.
//
// Lists: one warp per row stages it; when the list's nodes and the next one have
// distinct distances the warp extracts them by repeated warp minima, otherwise
// its first lane runs the reference's quicksort (middle pivot swapped to the
// left end, Lomuto partition with strict <, both halves recursed) on its row in
// shared memory.  Only positions below the list depth
// are needed, so ranges starting at or beyond it are skipped; the ranges are
// disjoint, so the order they are processed in does not matter and the
// smaller one goes first (explicit stack of at most log2(n) + 1 entries).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/cvrp_aco.h"
#include "aco_device.cuh"
#include "kernels.h"

namespace aco {
namespace {

__device__ __forceinline__ float dist_of(const float *x, const float *y, int type, int i, int j)
{
    const float dx = __fsub_rn(x[i], x[j]), dy = __fsub_rn(y[i], y[j]);
    const float s = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    if (type == ACO_DIST_CEIL_2D) return (float)(int)ceilf(__fsqrt_rn(s));
    if (type == ACO_DIST_ATT) {
        const float r = (float)__dsqrt_rn(__ddiv_rn((double)s, 10.0));
        const float t = (float)(int)r;
        return (float)(t < r ? (int)t + 1 : (int)t);
    }
    return __fsqrt_rn(s);
}

__global__ void dist_kernel(int n, const float *x, const float *y, int type, float *dist, int ld)
{
    const size_t total = (size_t)n * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / n), j = (int)(e - (size_t)i * n);
        dist[(size_t)i * ld + j] = dist_of(x, y, type, i, j);
    }
}

constexpr int kStack = 40;

// The reference's quicksort (utilities.cpp:246-266) on one row, stopping below `depth`.
__device__ void sort_row(float *v, int *idx, int n, int depth, int *status)
{
    int sl[kStack], sr[kStack], top = 0;
    sl[0] = 0;
    sr[0] = n - 1;
    top = 1;
    while (top > 0) {
        top--;
        const int l = sl[top], r = sr[top];
        if (l >= r || l >= depth) continue;
        const int m = (l + r) / 2;
        float tv = v[l]; v[l] = v[m]; v[m] = tv;
        int ti = idx[l]; idx[l] = idx[m]; idx[m] = ti;
        int last = l;
        const float pv = v[l];
        for (int k = l + 1; k <= r; k++)
            if (v[k] < pv) {
                ++last;
                tv = v[last]; v[last] = v[k]; v[k] = tv;
                ti = idx[last]; idx[last] = idx[k]; idx[k] = ti;
            }
        tv = v[l]; v[l] = v[last]; v[last] = tv;
        ti = idx[l]; idx[l] = idx[last]; idx[last] = ti;
        // ranges [l, last] and [last+1, r]: push the larger first
        const bool left_small = (last - l) <= (r - last - 1);
        if (top + 2 > kStack) { // cannot happen (depth <= log2(n) + 1); report rather than overflow
            if (status) atomicCAS(status, 0, ACO_ERR_CAPACITY);
            return;
        }
        if (left_small) {
            sl[top] = last + 1; sr[top] = r; top++;
            sl[top] = l; sr[top] = last; top++;
        } else {
            sl[top] = l; sr[top] = last; top++;
            sl[top] = last + 1; sr[top] = r; top++;
        }
    }
}

// The first `depth` entries of a staged row's list, warp-wide.  When the
// depth + 1 smallest values are all distinct, every correct sort puts the same
// nodes in the first depth positions, so the warp extracts them in depth + 1
// rounds of a 64-bit warp minimum over (value bits, index) -- for values from
// +0 to +inf the bits order as the floats.  Otherwise (a tie decides which node
// comes first, as with integer coordinates, or a row holds a negative value,
// -0 or NaN) lane 0 runs the reference's quicksort,
// whose partition order settles ties exactly as the host's.  On return idx[0,
// depth) holds the list.
__device__ void row_list(float *v, int *idx, int n, int depth, int lane, int *status)
{
    const unsigned FULLM = 0xffffffffu;
    if (depth < 32) {
        unsigned long long prev = 0ull, mine = ~0ull;
        bool first = true, odd = false; // odd: a negative value, -0 or NaN (their bits do not order as the floats)
        for (int r = 0; r <= depth; r++) {
            unsigned long long best = ~0ull;
            for (int i = lane; i < n; i += 32) {
                const uint32_t b = __float_as_uint(v[i]);
                if (first) odd = odd || b > 0x7f800000u;
                const unsigned long long k = ((unsigned long long)b << 32) | (unsigned)i;
                if ((first || k > prev) && k < best) best = k;
            }
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long w = __shfl_xor_sync(FULLM, best, o);
                best = w < best ? w : best;
            }
            if (lane == r) mine = best;
            prev = best;
            first = false;
        }
        // lanes 0..depth hold the depth + 1 smallest in order: a tie among them ends the fast path
        const unsigned nxt = __shfl_down_sync(FULLM, (unsigned)(mine >> 32), 1);
        const bool tie = lane < depth && (unsigned)(mine >> 32) == nxt;
        if (!__any_sync(FULLM, tie || odd)) {
            if (lane < depth) idx[lane] = (int)(mine & 0xffffffffu);
            __syncwarp();
            return;
        }
    }
    if (lane == 0) sort_row(v, idx, n, depth, status);
    __syncwarp();
}

// One warp per row: the lanes stage the row and pick its list (row_list), the
// lanes write the list.
__global__ void nn_kernel(int n, const float *dist, int ld, int depth, int rows_per_cta, int *nn, int *status)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * rows_per_cta + w;
    if (w >= rows_per_cta || row >= n) return;
    float *v = reinterpret_cast<float *>(sm) + (size_t)w * 2 * n;
    int *idx = reinterpret_cast<int *>(v + n);
    for (int i = lane; i < n; i += 32) {
        v[i] = dist[(size_t)row * ld + i];
        idx[i] = i;
    }
    __syncwarp();
    if (lane == 0) {
        v[row] = __int_as_float(0x7f800000); // the node itself and the depot never make the list
        v[0] = __int_as_float(0x7f800000);
    }
    __syncwarp();
    row_list(v, idx, n, depth, lane, status);
    for (int i = lane; i < depth; i += 32) nn[(size_t)row * depth + i] = idx[i];
}


// Distances of every instance's rows, a warp per row (same bits as dist_kernel).
__global__ void dist_rows_kernel(const PrepArgs *pa, const int *row_base, const int *row_inst, int total_rows)
{
    const int lane = threadIdx.x & 31;
    const int w0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int g = w0; g < total_rows; g += nw) {
        const int b = row_inst[g];
        const PrepArgs &a = pa[b];
        if (!a.device_prep) continue;
        const int i = g - row_base[b];
        float *row = a.dist + (size_t)i * a.ld;
        for (int j = lane; j < a.n; j += 32) row[j] = dist_of(a.x, a.y, a.dist_type, i, j);
    }
}

// Lists and tables of every instance's rows: a warp per row stages it and picks
// its list (row_list, as nn_kernel), and the lanes write the candidate tables
// (first K, padded with node 0 to Kp; demand in the high half of cand32) and
// the 2-opt list (first nn_ls) straight from the list.
__global__ void lists_rows_kernel(const PrepArgs *pa, const int *row_base, const int *row_inst, int total_rows,
                                  int rows_per_cta, int n_max, int *status)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *v = reinterpret_cast<float *>(sm) + (size_t)w * 2 * n_max;
    int *idx = reinterpret_cast<int *>(v + n_max);
    for (int g = blockIdx.x * rows_per_cta + w; g < total_rows; g += gridDim.x * rows_per_cta) {
        const int b = row_inst[g];
        const PrepArgs &a = pa[b];
        if (!a.device_prep || a.depth <= 0) continue;
        const int n = a.n, i = g - row_base[b];
        for (int k = lane; k < n; k += 32) {
            v[k] = a.dist[(size_t)i * a.ld + k];
            idx[k] = k;
        }
        __syncwarp();
        if (lane == 0) {
            v[i] = __int_as_float(0x7f800000); // the node itself and the depot never make the list
            v[0] = __int_as_float(0x7f800000);
        }
        __syncwarp();
        row_list(v, idx, n, a.depth, lane, status);
        for (int j = lane; j < a.Kp; j += 32) {
            const int c = j < a.K ? idx[j] : 0;
            a.nn16[(size_t)i * a.Kp + j] = (uint16_t)c;
            a.cand32[(size_t)i * a.Kp + j] = (uint32_t)c | ((uint32_t)(a.demand[c] & 0xFFFF) << 16);
        }
        for (int j = lane; j < a.nn_ls; j += 32) a.nnls[(size_t)i * a.nn_ls + j] = idx[j];
        __syncwarp(); // the row's buffers are reused by the warp's next row
    }
}

} // namespace

bool device_dist_supported(int dist_type) { return dist_type != ACO_DIST_GEO; }

size_t nn_rows_per_cta(int n)
{
    const size_t per_row = (size_t)8 * n;
    size_t rows = (size_t)(200 * 1024) / per_row;
    return std::min<size_t>(rows, 32);
}

cudaError_t launch_dist(int n, const float *x, const float *y, int dist_type, float *dist, int ld, int sm_count,
                        cudaStream_t st)
{
    const size_t total = (size_t)n * n;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)sm_count * 16);
    dist_kernel<<<std::max(blocks, 1), 256, 0, st>>>(n, x, y, dist_type, dist, ld);
    return cudaGetLastError();
}

cudaError_t launch_nn(int n, const float *dist, int ld, int depth, int *nn, int *status, cudaStream_t st)
{
    int rows = (int)nn_rows_per_cta(n);
    if (rows < 1) return cudaErrorInvalidValue;
    if (rows > 8) rows = 8; // warps (rows) per CTA
    const size_t smem = (size_t)rows * 8 * n;
    cudaError_t e = cudaFuncSetAttribute(nn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    nn_kernel<<<(n + rows - 1) / rows, 32 * rows, smem, st>>>(n, dist, ld, depth, rows, nn, status);
    return cudaGetLastError();
}

// The ants' lane seeds (g_aco.cpp:714-722): seed i = (int)(T0 + m (m + r_i) A)
// with m = i mod A and r_i the (i+1)-th ran01 draw from rnd_seed, in fp32 as
// written and converted as x86 cvttss2si does (NaN and out-of-range values give
// INT_MIN).  Draw i+1 is x0 * 16807^(i+1) mod (2^31 - 1), so every seed is
// computed independently.  Instance b of a batch draws from rnd_seed + b (int
// arithmetic, as the host adds it).
constexpr int kSeedRun = 16; // consecutive seeds of one ant a thread makes (nloc a multiple of it)

__global__ void seeds_kernel(const PrepArgs *pa, const int *ant_base, const int *ant_inst, long long runs, int nloc,
                             int seed_time, int rnd_seed)
{
    const float t0 = (float)seed_time;
    const int per_ant = nloc / kSeedRun;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < runs;
         e += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(e / per_ant), c = (int)(e - (long long)g * per_ant);
        const int b = ant_inst[g];
        const PrepArgs &a = pa[b];
        const long long i0 = (long long)(g - ant_base[b]) * nloc + (long long)c * kSeedRun;
        long long r = (long long)(int)((unsigned)rnd_seed + (unsigned)b) % 2147483647ll;
        if (r < 0) r += 2147483647ll;
        uint32_t x = pm_mul((uint32_t)r, pm_pow16807(i0 + 1)); // draw i0 + 1; the next ones one step apart
        const float av = (float)a.n_ants;
        for (int k = 0; k < kSeedRun; k++) {
            const long long i = i0 + k;
            const float m = (float)(int)(i % a.n_ants);
            const float v = __fadd_rn(t0, __fmul_rn(__fmul_rn(m, __fadd_rn(m, pm_uniform(x))), av));
            a.seeds[i] = (v >= -2147483648.0f && v < 2147483648.0f) ? __float2int_rz(v) : (int)0x80000000;
            x = pm_mul(x, 16807u);
        }
    }
}

// Scatter of staged uploads: piece k copies bytes [src_off, src_off + bytes)
// of the blob to dst.  The whole grid works on one piece after another, so a
// large piece (the seeds) spreads over every CTA.
__global__ void scatter_kernel(const ScatterPiece *pieces, int count, const unsigned char *blob)
{
    const unsigned long long t0 = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (int k = 0; k < count; k++) {
        const ScatterPiece pc = pieces[k];
        unsigned char *dst = reinterpret_cast<unsigned char *>(pc.dst);
        const unsigned char *src = blob + pc.src_off;
        const unsigned long long b = pc.bytes;
        if (((pc.dst | pc.src_off | b) & 15ull) == 0) {
            for (unsigned long long i = t0; i < b / 16; i += stride)
                reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
        } else if (((pc.dst | pc.src_off | b) & 3ull) == 0) {
            for (unsigned long long i = t0; i < b / 4; i += stride)
                reinterpret_cast<uint32_t *>(dst)[i] = reinterpret_cast<const uint32_t *>(src)[i];
        } else {
            for (unsigned long long i = t0; i < b; i += stride) dst[i] = src[i];
        }
    }
}

cudaError_t launch_scatter(const ScatterPiece *d_pieces, int count, const unsigned char *d_blob,
                           unsigned long long total_bytes, int sm_count, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    unsigned long long blocks = (total_bytes / 16 + 255) / 256;
    if (blocks > (unsigned long long)sm_count * 4) blocks = (unsigned long long)sm_count * 4;
    if (blocks < 1) blocks = 1;
    scatter_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_pieces, count, d_blob);
    return cudaGetLastError();
}

cudaError_t launch_prep_batch(const PrepArgs *d_args, const int *d_row_base, const int *d_row_inst, int total_rows,
                              int n_max, const int *d_ant_base, const int *d_ant_inst, int total_ants, int nloc,
                              int seed_time, int rnd_seed, int *status, int sm_count, cudaStream_t st)
{
    if (total_rows > 0) {
        const int blocks = std::min((total_rows + 7) / 8, sm_count * 8); // a warp per row, 8 a CTA
        dist_rows_kernel<<<std::max(blocks, 1), 256, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows);
        int rows = (int)nn_rows_per_cta(n_max);
        if (rows < 1) return cudaErrorInvalidValue;
        if (rows > 8) rows = 8;
        const size_t smem = (size_t)rows * 8 * n_max;
        cudaError_t e = cudaFuncSetAttribute(lists_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int lblocks = std::min((total_rows + rows - 1) / rows, sm_count * 16);
        lists_rows_kernel<<<std::max(lblocks, 1), 32 * rows, smem, st>>>(d_args, d_row_base, d_row_inst, total_rows,
                                                                         rows, n_max, status);
    }
    if (nloc % kSeedRun != 0) return cudaErrorInvalidValue;
    const long long runs = (long long)total_ants * (nloc / kSeedRun);
    if (runs > 0) {
        long long blocks = (runs + 255) / 256;
        if (blocks > sm_count * 8) blocks = sm_count * 8;
        seeds_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_args, d_ant_base, d_ant_inst, runs, nloc, seed_time, rnd_seed);
    }
    return cudaGetLastError();
}

} // namespace aco

using namespace aco;

extern "C" {

int aco_compute_distances_device(int n, const float *x, const float *y, int dist_type, float *dist, int ld,
                                 void *stream)
{
    if (n < 1 || !x || !y || !dist || ld < n || !device_dist_supported(dist_type)) return ACO_ERR_INVALID;
    int dev = 0, sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    return launch_dist(n, x, y, dist_type, dist, ld, sm, static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? ACO_OK
               : ACO_ERR_CUDA;
}

int aco_compute_nn_lists_device(int n, const float *dist, int ld, int nn_ls, int nn_ants, int *nn, int *depth,
                                void *stream)
{
    if (n < 2 || !dist || !depth || ld < n || nn_rows_per_cta(n) < 1) return ACO_ERR_INVALID;
    int d = nn_ls >= nn_ants ? nn_ls : nn_ants;
    if (d >= n) d = n - 1;
    if (d < 0) d = 0;
    *depth = d;
    if (d == 0) return ACO_OK;
    if (!nn) return ACO_ERR_INVALID;
    return launch_nn(n, dist, ld, d, nn, nullptr, static_cast<cudaStream_t>(stream)) == cudaSuccess ? ACO_OK
                                                                                                     : ACO_ERR_CUDA;
}

} // extern "C"
