// mpnn.cu -- the edge-scoring message-passing network of the learned prior:
// forward, backward and the Adam step, with every dense product on the
// tcgen05 tensor cores (BF16 operands, FP32 accumulation in tensor memory).
//
// Graph: node i has k out-edges, rows i*k .. i*k+k-1 of every edge array, to
// its k nearest customers (nbr).  Hidden width 64.  Per layer (the oracle in
// oracle/mpnn_oracle.py states the same equations in FP64):
//   P  = h W^T + b              node GEMM, N = 256 (U | V | B | C)
//   q  = e A^T + a + B_i + C_j  edge GEMM + gathers
//   e' = e + relu(q);  g = sigmoid(e')
//   u  = U + (1/k) sum_j g V_j;  h' = h + relu(u)
// Head: z = relu(e W_h^T + b_h), logit s = z . w_o + b_o; weighted BCE loss.
//
// Edge kernels work on tiles of floor(128/k) whole nodes (their edges are one
// contiguous row range), so the per-node sums need no atomics; the
// contributions to a neighbour's row (dV, dC) are float atomics.  Weight
// gradients accumulate in tensor memory across the tiles a persistent CTA
// processes and are added to the gradient buffer once per CTA.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "../../include/cvrp_aco.h"
#include "aco_device.cuh"
#include "umma.cuh"

namespace aco {
namespace {

constexpr int H = 64;
constexpr int FN = ACO_MPNN_NODE_FEATURES;
constexpr int TPB = 128; // 4 warps: thread t owns TMEM lane t / tile row t

// ---- packed parameter layout (same order as the oracle) --------------------
struct ParamOffsets {
    int W_n, b_n, W_e, b_e;
    int W[8], b[8], A[8], a[8];
    int W_h, b_h, w_o, b_o, count;
};

__host__ __device__ inline ParamOffsets param_offsets(int L)
{
    ParamOffsets o{};
    int p = 0;
    o.W_n = p; p += H * FN;
    o.b_n = p; p += H;
    o.W_e = p; p += H;
    o.b_e = p; p += H;
    for (int l = 0; l < L; l++) {
        o.W[l] = p; p += 4 * H * H;
        o.b[l] = p; p += 4 * H;
        o.A[l] = p; p += H * H;
        o.a[l] = p; p += H;
    }
    o.W_h = p; p += H * H;
    o.b_h = p; p += H;
    o.w_o = p; p += H;
    o.b_o = p; p += 1;
    o.count = p;
    return o;
}

// ---- workspace layout ------------------------------------------------------
struct Workspace {
    int *status;
    float *loss;
    float *h, *e, *P, *q, *u; // saved activations
    float *s;                  // edge logits
    float *dh, *de, *dP;       // backward
    size_t bytes;
};

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

Workspace carve(void *base, int N, int k, int L)
{
    const size_t E = (size_t)N * k;
    Workspace w{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = al256(off + bytes);
        return o;
    };
    const size_t o_status = take(64), o_loss = take(64);
    const size_t o_h = take(sizeof(float) * (L + 1) * N * H), o_e = take(sizeof(float) * (L + 1) * E * H);
    const size_t o_P = take(sizeof(float) * L * N * 4 * H), o_q = take(sizeof(float) * L * E * H);
    const size_t o_u = take(sizeof(float) * L * N * H), o_s = take(sizeof(float) * E);
    const size_t o_dh = take(sizeof(float) * N * H), o_de = take(sizeof(float) * E * H);
    const size_t o_dP = take(sizeof(float) * N * 4 * H);
    w.bytes = off;
    if (base) {
        char *b = static_cast<char *>(base);
        w.status = (int *)(b + o_status);
        w.loss = (float *)(b + o_loss);
        w.h = (float *)(b + o_h);
        w.e = (float *)(b + o_e);
        w.P = (float *)(b + o_P);
        w.q = (float *)(b + o_q);
        w.u = (float *)(b + o_u);
        w.s = (float *)(b + o_s);
        w.dh = (float *)(b + o_dh);
        w.de = (float *)(b + o_de);
        w.dP = (float *)(b + o_dP);
    }
    return w;
}

// ---- device helpers ----------------------------------------------------------
__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }

// rows [0, R) x K of a row-major fp32 source (row stride ld) -> K-major bf16 tile;
// rows >= valid are zero.  K a multiple of 8.
__device__ void stage_rows(uint8_t *tile, const float *src, size_t ld, int R, int K, int valid)
{
    const int q = K >> 2;
    for (int idx = threadIdx.x; idx < R * q; idx += blockDim.x) {
        const int r = idx / q, c = (idx - r * q) << 2;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (r < valid) v = *reinterpret_cast<const float4 *>(src + (size_t)r * ld + c);
        const uint32_t lo = (uint32_t)umma::bf16_bits(v.x) | ((uint32_t)umma::bf16_bits(v.y) << 16);
        const uint32_t hi = (uint32_t)umma::bf16_bits(v.z) | ((uint32_t)umma::bf16_bits(v.w) << 16);
        *reinterpret_cast<uint2 *>(tile + umma::kmajor_offset(r, c, K)) = make_uint2(lo, hi);
    }
}

// Transposed staging: tile(n, kk) = src[kk * ld + n] for n < Rn, kk < Kk;
// source rows kk >= valid_k are zero.
__device__ void stage_cols(uint8_t *tile, const float *src, size_t ld, int Rn, int Kk, int valid_k)
{
    for (int idx = threadIdx.x; idx < Rn * Kk; idx += blockDim.x) {
        const int kk = idx / Rn, n = idx - kk * Rn;
        const float v = kk < valid_k ? src[(size_t)kk * ld + n] : 0.f;
        *reinterpret_cast<uint16_t *>(tile + umma::kmajor_offset(n, kk, Kk)) = umma::bf16_bits(v);
    }
}

// Zero rows [r0, R) of a K-major tile with K columns.
__device__ void zero_rows(uint8_t *tile, int r0, int R, int K)
{
    const int q = K >> 2;
    for (int idx = threadIdx.x; idx < (R - r0) * q; idx += blockDim.x) {
        const int r = r0 + idx / q, c = (idx % q) << 2;
        *reinterpret_cast<uint2 *>(tile + umma::kmajor_offset(r, c, K)) = make_uint2(0u, 0u);
    }
}

// One GEMM D(128 x N) (+)= A(128 x K) B(N x K)^T issued by thread 0.
__device__ __forceinline__ void gemm_issue(uint32_t tmem_d, const uint8_t *a, const uint8_t *b, int K, int N,
                                           bool accumulate)
{
    if (threadIdx.x == 0) {
        const uint32_t id = umma::idesc_bf16(128, N);
        const uint32_t aa = smem_u32(a), bb = smem_u32(b);
        for (int s = 0; s < (K >> 4); s++)
            umma::mma_bf16(tmem_d, umma::smem_desc(aa, K, s), umma::smem_desc(bb, K, s), id, accumulate || s > 0);
    }
}

// Make staged operands visible to the tensor core and the CTA.
__device__ __forceinline__ void operands_ready()
{
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}

// Commit the issued MMAs and wait for them (bounded).  Returns false (uniformly)
// on timeout after recording ACO_ERR_TIMEOUT.
__device__ bool gemm_wait(uint64_t *bar, uint32_t &phase, int *status)
{
    if (threadIdx.x == 0) umma::commit(bar);
    bool ok = mbar_wait(bar, phase);
    if (!ok) {
        set_status(status, ACO_ERR_TIMEOUT);
        mbar_wait(bar, phase); // let the MMAs in flight finish before the CTA lets go of its memory
    }
    phase ^= 1u;
    ok = !__syncthreads_or(!ok);
    umma::fence_after();
    return ok;
}

// Tensor-memory set-up shared by the kernels: mbarrier + allocation by warp 0.
__device__ void tmem_setup(uint64_t *bar, uint32_t *slot, uint32_t ncols)
{
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (threadIdx.x < 32) umma::tmem_alloc(slot, ncols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}

__device__ void tmem_teardown(uint32_t base, uint32_t ncols)
{
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    if (threadIdx.x < 32) umma::tmem_dealloc(base, ncols);
}

// Read this thread's 64 accumulator columns starting at column col0.
__device__ __forceinline__ void tmem_row64(uint32_t base, int col0, float (&v)[64])
{
    const int lane0 = (threadIdx.x >> 5) << 5;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float t[16];
        umma::tmem_ld16(umma::taddr(base, lane0, col0 + 16 * c), t);
#pragma unroll
        for (int i = 0; i < 16; i++) v[16 * c + i] = t[i];
    }
}

// ---- forward -----------------------------------------------------------------
__global__ void embed_kernel(int N, int k, const float *prm, ParamOffsets o, const float *nf, const float *ef,
                             float *h0, float *e0)
{
    const size_t NH = (size_t)N * H, EH = (size_t)N * k * H;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < NH + EH;
         idx += (size_t)gridDim.x * blockDim.x) {
        if (idx < NH) {
            const size_t i = idx / H;
            const int c = (int)(idx % H);
            float acc = 0.f;
            for (int f = 0; f < FN; f++) acc = __fmaf_rn(prm[o.W_n + c * FN + f], nf[i * FN + f], acc);
            h0[idx] = acc + prm[o.b_n + c];
        } else {
            const size_t j = idx - NH, ei = j / H;
            const int c = (int)(j % H);
            e0[j] = __fmaf_rn(prm[o.W_e + c], ef[ei], prm[o.b_e + c]);
        }
    }
}

// P = h W^T + b: tiles of 128 nodes, N = 256.
struct NodeGemmSmem {
    static constexpr size_t A = 0, B = A + 128 * H * 2, BYTES = B + 4 * H * H * 2;
};

__global__ void __launch_bounds__(TPB) node_gemm_kernel(int N, const float *h, const float *W, const float *bias,
                                                        float *P, int *status)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    uint8_t *As = sm + NodeGemmSmem::A, *Bs = sm + NodeGemmSmem::B;
    tmem_setup(&bar, &slot, 256);
    const uint32_t tm = slot;
    uint32_t phase = 0;
    stage_rows(Bs, W, H, 4 * H, H, 4 * H);
    const int tiles = (N + 127) / 128;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int r0 = t * 128, valid = min(128, N - r0);
        stage_rows(As, h + (size_t)r0 * H, H, 128, H, valid);
        operands_ready();
        gemm_issue(tm, As, Bs, H, 4 * H, false);
        if (!gemm_wait(&bar, phase, status)) break;
        const int r = threadIdx.x, lane0 = (threadIdx.x >> 5) << 5;
        for (int c = 0; c < 16; c++) {
            float v[16];
            umma::tmem_ld16(umma::taddr(tm, lane0, 16 * c), v);
            if (r < valid) {
                float *dst = P + (size_t)(r0 + r) * 4 * H + 16 * c;
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4 *>(dst + i) =
                        make_float4(v[i] + bias[16 * c + i], v[i + 1] + bias[16 * c + i + 1],
                                    v[i + 2] + bias[16 * c + i + 2], v[i + 3] + bias[16 * c + i + 3]);
            }
        }
        umma::fence_before();
        __syncthreads();
    }
    tmem_teardown(tm, 256);
}

// Edge layer forward on tiles of npt = 128/k nodes.  M: the tile's 128 rows of
// 64 fp32 values at row stride MS (the accumulator, then the gated messages),
// padded so that the TMEM-lane-per-row writes fall in distinct banks.
constexpr int MS = H + 1;
struct EdgeFwdSmem {
    static constexpr size_t A = 0, B = A + 128 * H * 2, M = B + H * H * 2, BYTES = M + 128 * MS * 4;
};

__global__ void __launch_bounds__(TPB) edge_fwd_kernel(int N, int k, const float *Wt, const float *a_bias,
                                                       const float *e_in, const float *P, const float *h_in,
                                                       const int *nbr, float *q_out, float *e_out, float *u_out,
                                                       float *h_out, int *status)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    uint8_t *As = sm + EdgeFwdSmem::A, *Bs = sm + EdgeFwdSmem::B;
    float *ms = reinterpret_cast<float *>(sm + EdgeFwdSmem::M);
    tmem_setup(&bar, &slot, 64);
    const uint32_t tm = slot;
    uint32_t phase = 0;
    stage_rows(Bs, Wt, H, H, H, H); // A_l[o][i]: rows o, K = i
    const int npt = 128 / k, tiles = (N + npt - 1) / npt;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int n0 = t * npt, nodes = min(npt, N - n0), rows = nodes * k;
        const size_t e0 = (size_t)n0 * k;
        stage_rows(As, e_in + e0 * H, H, 128, H, rows);
        operands_ready();
        gemm_issue(tm, As, Bs, H, H, false);
        if (!gemm_wait(&bar, phase, status)) break;
        {   // the accumulator rows into shared memory (thread r holds TMEM lane r = row r)
            const int r = threadIdx.x;
            float d[64];
            tmem_row64(tm, 0, d);
#pragma unroll
            for (int c = 0; c < H; c++) ms[r * MS + c] = d[c];
        }
        __syncthreads();
        // epilogue by rows: a warp takes row r, lane l its channels 2l, 2l+1, so every
        // global access of e, q and the P rows is one coalesced 256-byte row
        {
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, c = 2 * lane;
            const float2 ab = *reinterpret_cast<const float2 *>(a_bias + c);
            for (int r = warp; r < rows; r += TPB / 32) {
                const size_t ei = e0 + r;
                const int src = n0 + r / k;
                int j = nbr[ei];
                if ((unsigned)j >= (unsigned)N) { // a neighbour id outside the batch: report, read node 0
                    if (lane == 0) set_status(status, ACO_ERR_INVALID);
                    j = 0;
                }
                const float *Pi = P + (size_t)src * 4 * H, *Pj = P + (size_t)j * 4 * H;
                const float2 pi = *reinterpret_cast<const float2 *>(Pi + 2 * H + c);
                const float2 pj = *reinterpret_cast<const float2 *>(Pj + 3 * H + c);
                const float2 vj = *reinterpret_cast<const float2 *>(Pj + H + c);
                const float2 ein = *reinterpret_cast<const float2 *>(e_in + ei * H + c);
                float *mr = ms + r * MS + c;
                const float q0 = mr[0] + ab.x + pi.x + pj.x, q1 = mr[1] + ab.y + pi.y + pj.y;
                const float en0 = ein.x + fmaxf(q0, 0.f), en1 = ein.y + fmaxf(q1, 0.f);
                *reinterpret_cast<float2 *>(q_out + ei * H + c) = make_float2(q0, q1);
                *reinterpret_cast<float2 *>(e_out + ei * H + c) = make_float2(en0, en1);
                mr[0] = sigmoidf_(en0) * vj.x; // the gated message replaces the accumulator
                mr[1] = sigmoidf_(en1) * vj.y;
            }
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < nodes * H; idx += blockDim.x) {
            const int qn = idx / H, c = idx - qn * H, i = n0 + qn;
            float acc = 0.f;
            for (int j = 0; j < k; j++) acc += ms[(qn * k + j) * MS + c];
            const float uv = P[(size_t)i * 4 * H + c] + acc / (float)k;
            u_out[(size_t)i * H + c] = uv;
            h_out[(size_t)i * H + c] = h_in[(size_t)i * H + c] + fmaxf(uv, 0.f);
        }
        umma::fence_before();
        __syncthreads();
    }
    tmem_teardown(tm, 64);
}

// Head (tiles of 128 edges).  Inference: logits only.  Training: also the
// weighted BCE loss, dL/ds, dz, de = dz W_h and the head's weight gradients.
struct HeadSmem {
    static constexpr size_t A = 0, B = A + 128 * H * 2, BT = B + H * H * 2, DZ = BT + H * H * 2,
                            DZT = DZ + 128 * H * 2, ET = DZT + 128 * 128 * 2, RED = ET + H * 128 * 2,
                            BYTES = RED + 4 * H * 4;
};

__global__ void __launch_bounds__(TPB) head_kernel(size_t E, const float *prm, ParamOffsets o, const float *eL,
                                                   float *s_out, const float *labels, float pos_weight, float inv_E,
                                                   float *de, float *grad, float *loss, int *status)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    const bool train = labels != nullptr;
    uint8_t *As = sm + HeadSmem::A, *Bs = sm + HeadSmem::B, *BTs = sm + HeadSmem::BT, *DZs = sm + HeadSmem::DZ;
    uint8_t *DZTs = sm + HeadSmem::DZT, *ETs = sm + HeadSmem::ET;
    float *red = reinterpret_cast<float *>(sm + HeadSmem::RED); // b_h (64), w_o (64), b_o, loss
    tmem_setup(&bar, &slot, 256);
    const uint32_t tm = slot; // cols 0-63 z, 64-127 de, 128-191 dW_h
    uint32_t phase = 0;
    const float *Wh = prm + o.W_h, *bh = prm + o.b_h, *wo = prm + o.w_o;
    const float bo = prm[o.b_o];
    stage_rows(Bs, Wh, H, H, H, H);      // W_h[o][i]
    if (train) {
        stage_cols(BTs, Wh, H, H, H, H); // tile(i, o) = W_h[o][i]
        zero_rows(DZTs, H, 128, 128);    // rows o >= 64 of the transposed dz stay zero
        for (int i = threadIdx.x; i < 4 * H; i += blockDim.x) red[i] = 0.f;
    }
    bool wg_started = false;
    const size_t tiles = (E + 127) / 128;
    for (size_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const size_t e0 = t * 128;
        const int rows = (int)min((size_t)128, E - e0);
        stage_rows(As, eL + e0 * H, H, 128, H, rows);
        if (train) stage_cols(ETs, eL + e0 * H, H, H, 128, rows); // tile(i, e) = eL[e][i]
        operands_ready();
        gemm_issue(tm, As, Bs, H, H, false);
        if (!gemm_wait(&bar, phase, status)) break;
        const int r = threadIdx.x;
        float zp[64];
        tmem_row64(tm, 0, zp);
        float sv = bo;
        for (int c = 0; c < H; c++) {
            zp[c] += bh[c];
            sv += fmaxf(zp[c], 0.f) * wo[c];
        }
        if (r < rows) s_out[e0 + r] = sv;
        if (!train) {
            umma::fence_before();
            __syncthreads();
            continue;
        }
        float ds = 0.f;
        if (r < rows) {
            const float y = labels[e0 + r];
            const float sg = sigmoidf_(sv);
            // -(w y log sig(s) + (1-y) log(1-sig(s))), with log sig(s) = -softplus(-s)
            const float sp_neg = fmaxf(-sv, 0.f) + log1pf(expf(-fabsf(sv)));
            const float sp_pos = fmaxf(sv, 0.f) + log1pf(expf(-fabsf(sv)));
            atomicAdd(&red[4 * H - 1], (pos_weight * y * sp_neg + (1.f - y) * sp_pos) * inv_E);
            ds = (pos_weight * y * (sg - 1.f) + (1.f - y) * sg) * inv_E;
            atomicAdd(&red[2 * H], ds);
        }
        for (int c = 0; c < H; c++) {
            const float z = fmaxf(zp[c], 0.f);
            const float dz = zp[c] > 0.f ? ds * wo[c] : 0.f;
            if (r < rows) {
                atomicAdd(&red[c], dz);
                atomicAdd(&red[H + c], ds * z);
            }
            *reinterpret_cast<uint16_t *>(DZs + umma::kmajor_offset(r, c, H)) = umma::bf16_bits(dz);
            *reinterpret_cast<uint16_t *>(DZTs + umma::kmajor_offset(c, r, 128)) = umma::bf16_bits(dz);
        }
        operands_ready();
        gemm_issue(tm + 64, DZs, BTs, H, H, false);         // de = dz W_h
        gemm_issue(tm + 128, DZTs, ETs, 128, H, wg_started); // dW_h += dz^T eL
        wg_started = true;
        if (!gemm_wait(&bar, phase, status)) break;
        float dv[64];
        tmem_row64(tm, 64, dv);
        if (r < rows)
            for (int c = 0; c < H; c += 4)
                *reinterpret_cast<float4 *>(de + (e0 + r) * H + c) = make_float4(dv[c], dv[c + 1], dv[c + 2], dv[c + 3]);
        umma::fence_before();
        __syncthreads();
    }
    if (train) {
        __syncthreads();
        if (wg_started) { // rows o < 64 of the accumulated dW_h (TMEM lanes 0-63)
            float w[64];
            tmem_row64(tm, 128, w);
            if (threadIdx.x < H)
                for (int c = 0; c < H; c++) atomicAdd(&grad[o.W_h + threadIdx.x * H + c], w[c]);
        }
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            atomicAdd(&grad[o.b_h + i], red[i]);
            atomicAdd(&grad[o.w_o + i], red[H + i]);
        }
        if (threadIdx.x == 0) {
            atomicAdd(&grad[o.b_o], red[2 * H]);
            atomicAdd(loss, red[4 * H - 1]);
        }
    }
    tmem_teardown(tm, 256);
}

// ---- backward ------------------------------------------------------------------
// Edge layer backward on node tiles.  dh = dL/dh', de = dL/de' (overwritten by
// dL/de); dP receives du (owned), dV (atomic), dB (owned), dC (atomic).
struct EdgeBwdSmem {
    static constexpr size_t DQ = 0, BT = DQ + 128 * H * 2, DQT = BT + H * H * 2, ET = DQT + 128 * 128 * 2,
                            DU = ET + H * 128 * 2, DQF = DU + 128 * H * 4, RED = DQF + 128 * H * 4,
                            BYTES = RED + H * 4;
};

__global__ void __launch_bounds__(TPB) edge_bwd_kernel(int N, int k, const float *A_w, const float *P,
                                                       const float *u, const float *q, const float *e_in,
                                                       const float *e_out, const int *nbr, const float *dh, float *de,
                                                       float *dP, float *gA, float *ga, int *status)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    uint8_t *DQs = sm + EdgeBwdSmem::DQ, *BTs = sm + EdgeBwdSmem::BT, *DQTs = sm + EdgeBwdSmem::DQT;
    uint8_t *ETs = sm + EdgeBwdSmem::ET;
    float *dus = reinterpret_cast<float *>(sm + EdgeBwdSmem::DU);  // npt x 64
    float *dqf = reinterpret_cast<float *>(sm + EdgeBwdSmem::DQF); // 128 x 64
    float *red = reinterpret_cast<float *>(sm + EdgeBwdSmem::RED); // grad of a
    tmem_setup(&bar, &slot, 128);
    const uint32_t tm = slot; // cols 0-63 dgrad, 64-127 dA
    uint32_t phase = 0;
    stage_cols(BTs, A_w, H, H, H, H); // tile(i, o) = A[o][i]
    zero_rows(DQTs, H, 128, 128);
    for (int i = threadIdx.x; i < H; i += blockDim.x) red[i] = 0.f;
    bool wg_started = false;
    const int npt = 128 / k, tiles = (N + npt - 1) / npt;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int n0 = t * npt, nodes = min(npt, N - n0), rows = nodes * k;
        const size_t e0 = (size_t)n0 * k;
        for (int idx = threadIdx.x; idx < nodes * H; idx += blockDim.x) {
            const int qn = idx / H, c = idx - qn * H, i = n0 + qn;
            const float dv = u[(size_t)i * H + c] > 0.f ? dh[(size_t)i * H + c] : 0.f;
            dus[qn * H + c] = dv;
            dP[(size_t)i * 4 * H + c] = dv;
        }
        stage_cols(ETs, e_in + e0 * H, H, H, 128, rows); // tile(i, e) = e_in[e][i]
        __syncthreads();
        const int r = threadIdx.x;
        if (r < rows) {
            const size_t ei = e0 + r;
            const int ql = r / k;
            int j = nbr[ei];
            if ((unsigned)j >= (unsigned)N) {
                set_status(status, ACO_ERR_INVALID);
                j = 0;
            }
            const float *Pj = P + (size_t)j * 4 * H;
            for (int c = 0; c < H; c++) {
                const float due = dus[ql * H + c] / (float)k;
                const float g = sigmoidf_(e_out[ei * H + c]);
                atomicAdd(&dP[(size_t)j * 4 * H + H + c], due * g);
                const float dt = de[ei * H + c] + due * Pj[H + c] * g * (1.f - g);
                const float dq = q[ei * H + c] > 0.f ? dt : 0.f;
                de[ei * H + c] = dt; // the residual part; the GEMM part is added below
                dqf[r * H + c] = dq;
                atomicAdd(&dP[(size_t)j * 4 * H + 3 * H + c], dq);
                *reinterpret_cast<uint16_t *>(DQs + umma::kmajor_offset(r, c, H)) = umma::bf16_bits(dq);
                *reinterpret_cast<uint16_t *>(DQTs + umma::kmajor_offset(c, r, 128)) = umma::bf16_bits(dq);
            }
        } else {
            for (int c = 0; c < H; c++) {
                dqf[r * H + c] = 0.f;
                *reinterpret_cast<uint16_t *>(DQs + umma::kmajor_offset(r, c, H)) = 0;
                *reinterpret_cast<uint16_t *>(DQTs + umma::kmajor_offset(c, r, 128)) = 0;
            }
        }
        operands_ready();
        gemm_issue(tm, DQs, BTs, H, H, false);             // dq A
        gemm_issue(tm + 64, DQTs, ETs, 128, H, wg_started); // dA += dq^T e_in
        wg_started = true;
        if (!gemm_wait(&bar, phase, status)) break;
        float dv[64];
        tmem_row64(tm, 0, dv);
        if (r < rows) {
            const size_t ei = e0 + r;
            for (int c = 0; c < H; c++) de[ei * H + c] += dv[c];
        }
        for (int idx = threadIdx.x; idx < nodes * H; idx += blockDim.x) {
            const int qn = idx / H, c = idx - qn * H;
            float acc = 0.f;
            for (int jj = 0; jj < k; jj++) acc += dqf[(qn * k + jj) * H + c];
            dP[(size_t)(n0 + qn) * 4 * H + 2 * H + c] = acc;
        }
        for (int c = threadIdx.x; c < H; c += blockDim.x) {
            float acc = 0.f;
            for (int rr = 0; rr < rows; rr++) acc += dqf[rr * H + c];
            red[c] += acc;
        }
        umma::fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (wg_started) {
        float w[64];
        tmem_row64(tm, 64, w);
        if (threadIdx.x < H)
            for (int c = 0; c < H; c++) atomicAdd(&gA[threadIdx.x * H + c], w[c]);
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) atomicAdd(&ga[i], red[i]);
    tmem_teardown(tm, 128);
}

// dh += dP W (K = 256), dW += dP^T h (two M = 128 halves), db += sum dP.
struct NodeBwdSmem {
    static constexpr size_t A = 0, BT = A + 128 * 4 * H * 2, AT = BT + H * 4 * H * 2, HT = AT + 2 * 128 * 128 * 2,
                            RED = HT + H * 128 * 2, BYTES = RED + 4 * H * 4;
};

__global__ void __launch_bounds__(TPB) node_bwd_kernel(int N, const float *W, const float *h_in, const float *dP,
                                                       float *dh, float *gW, float *gb, int *status)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    uint8_t *As = sm + NodeBwdSmem::A, *BTs = sm + NodeBwdSmem::BT, *ATs = sm + NodeBwdSmem::AT;
    uint8_t *HTs = sm + NodeBwdSmem::HT;
    float *red = reinterpret_cast<float *>(sm + NodeBwdSmem::RED);
    tmem_setup(&bar, &slot, 256);
    const uint32_t tm = slot; // 0-63 dgrad, 64-127 dW rows 0-127, 128-191 dW rows 128-255
    uint32_t phase = 0;
    stage_cols(BTs, W, H, H, 4 * H, 4 * H); // tile(c, o) = W[o][c]
    for (int i = threadIdx.x; i < 4 * H; i += blockDim.x) red[i] = 0.f;
    bool wg_started = false;
    const int tiles = (N + 127) / 128;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int r0 = t * 128, valid = min(128, N - r0);
        stage_rows(As, dP + (size_t)r0 * 4 * H, 4 * H, 128, 4 * H, valid);
        stage_cols(ATs, dP + (size_t)r0 * 4 * H, 4 * H, 128, 128, valid);                 // tile(o, i) = dP[i][o], o < 128
        stage_cols(ATs + 128 * 128 * 2, dP + (size_t)r0 * 4 * H + 128, 4 * H, 128, 128, valid); // o in [128, 256)
        stage_cols(HTs, h_in + (size_t)r0 * H, H, H, 128, valid);                       // tile(c, i) = h[i][c]
        for (int oo = threadIdx.x; oo < 4 * H; oo += blockDim.x) {
            float acc = 0.f;
            for (int i = 0; i < valid; i++) acc += dP[(size_t)(r0 + i) * 4 * H + oo];
            red[oo] += acc;
        }
        operands_ready();
        gemm_issue(tm, As, BTs, 4 * H, H, false);
        gemm_issue(tm + 64, ATs, HTs, 128, H, wg_started);
        gemm_issue(tm + 128, ATs + 128 * 128 * 2, HTs, 128, H, wg_started);
        wg_started = true;
        if (!gemm_wait(&bar, phase, status)) break;
        float dv[64];
        tmem_row64(tm, 0, dv);
        const int r = threadIdx.x;
        if (r < valid)
            for (int c = 0; c < H; c++) dh[(size_t)(r0 + r) * H + c] += dv[c];
        umma::fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (wg_started) {
        float w0[64], w1[64];
        tmem_row64(tm, 64, w0);
        tmem_row64(tm, 128, w1);
        const int o = threadIdx.x;
        for (int c = 0; c < H; c++) {
            atomicAdd(&gW[o * H + c], w0[c]);
            atomicAdd(&gW[(128 + o) * H + c], w1[c]);
        }
    }
    for (int i = threadIdx.x; i < 4 * H; i += blockDim.x) atomicAdd(&gb[i], red[i]);
    tmem_teardown(tm, 256);
}

// Input embeddings' gradients (CUDA cores: K = 5 and 1).
__global__ void embed_bwd_kernel(int N, int k, ParamOffsets o, const float *nf, const float *ef, const float *dh0,
                                 const float *de0, float *grad)
{
    // each block: one output channel c, all nodes / edges
    const int c = blockIdx.x;
    __shared__ float red[8][FN + 3];
    float acc[FN + 3] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const float d = dh0[(size_t)i * H + c];
        for (int f = 0; f < FN; f++) acc[f] += d * nf[(size_t)i * FN + f];
        acc[FN] += d;
    }
    const size_t E = (size_t)N * k;
    for (size_t e = threadIdx.x; e < E; e += blockDim.x) {
        const float d = de0[e * H + c];
        acc[FN + 1] += d * ef[e];
        acc[FN + 2] += d;
    }
    for (int f = 0; f < FN + 3; f++)
        for (int off = 16; off > 0; off >>= 1) acc[f] += __shfl_xor_sync(0xffffffffu, acc[f], off);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int f = 0; f < FN + 3; f++) red[w][f] = acc[f];
    __syncthreads();
    if (threadIdx.x < FN + 3) {
        float s = 0.f;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) s += red[ww][threadIdx.x];
        const int f = threadIdx.x;
        if (f < FN) grad[o.W_n + c * FN + f] = s;
        else if (f == FN) grad[o.b_n + c] = s;
        else if (f == FN + 1) grad[o.W_e + c] = s;
        else grad[o.b_e + c] = s;
    }
}

__global__ void adam_kernel(int n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                            float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int g_sm_count = 0;

int sm_count()
{
    if (g_sm_count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 148;
    }
    return g_sm_count;
}

template <typename K>
cudaError_t set_smem(K kern, size_t bytes)
{
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

bool args_ok(int N, int k, int L)
{
    return N >= 1 && k >= 1 && k <= 32 && L >= 1 && L <= 8 && (size_t)N * k < ((size_t)1 << 31);
}

int run_forward(int N, int k, int L, const float *prm, const float *nf, const float *ef, const int *nbr,
                const Workspace &w, cudaStream_t st)
{
    const ParamOffsets o = param_offsets(L);
    const size_t E = (size_t)N * k;
    const int grid_sm = sm_count() * 2;
    embed_kernel<<<std::min<size_t>(((size_t)N * H + E * H + 255) / 256, (size_t)grid_sm * 8), 256, 0, st>>>(
        N, k, prm, o, nf, ef, w.h, w.e);
    if (set_smem(node_gemm_kernel, NodeGemmSmem::BYTES) != cudaSuccess) return ACO_ERR_CUDA;
    if (set_smem(edge_fwd_kernel, EdgeFwdSmem::BYTES) != cudaSuccess) return ACO_ERR_CUDA;
    const int ntiles = (N + 127) / 128, npt = 128 / k, etiles = (N + npt - 1) / npt;
    for (int l = 0; l < L; l++) {
        const float *h = w.h + (size_t)l * N * H, *e = w.e + (size_t)l * E * H;
        float *P = w.P + (size_t)l * N * 4 * H;
        node_gemm_kernel<<<std::min(ntiles, grid_sm), TPB, NodeGemmSmem::BYTES, st>>>(N, h, prm + o.W[l],
                                                                                     prm + o.b[l], P, w.status);
        edge_fwd_kernel<<<std::min(etiles, grid_sm), TPB, EdgeFwdSmem::BYTES, st>>>(
            N, k, prm + o.A[l], prm + o.a[l], e, P, h, nbr, w.q + (size_t)l * E * H, w.e + (size_t)(l + 1) * E * H,
            w.u + (size_t)l * N * H, w.h + (size_t)(l + 1) * N * H, w.status);
    }
    return cudaGetLastError() == cudaSuccess ? ACO_OK : ACO_ERR_CUDA;
}

} // namespace
} // namespace aco

using namespace aco;

extern "C" {

int aco_mpnn_param_count(int layers)
{
    if (layers < 1 || layers > 8) return ACO_ERR_INVALID;
    return param_offsets(layers).count;
}

int aco_mpnn_workspace_bytes(int n_nodes, int k, int layers, size_t *bytes)
{
    if (!bytes || !args_ok(n_nodes, k, layers)) return ACO_ERR_INVALID;
    *bytes = carve(nullptr, n_nodes, k, layers).bytes;
    return ACO_OK;
}

int aco_mpnn_forward(int n_nodes, int k, int layers, const float *params, const float *node_feat,
                     const float *edge_feat, const int *nbr, void *workspace, size_t ws_bytes, float *scores,
                     void *stream)
{
    if (!args_ok(n_nodes, k, layers) || !params || !node_feat || !edge_feat || !nbr || !workspace || !scores)
        return ACO_ERR_INVALID;
    const Workspace w = carve(workspace, n_nodes, k, layers);
    if (ws_bytes < w.bytes) return ACO_ERR_CAPACITY;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(w.status, 0, 64, st) != cudaSuccess) return ACO_ERR_CUDA;
    int rc = run_forward(n_nodes, k, layers, params, node_feat, edge_feat, nbr, w, st);
    if (rc != ACO_OK) return rc;
    const ParamOffsets o = param_offsets(layers);
    const size_t E = (size_t)n_nodes * k;
    if (set_smem(head_kernel, HeadSmem::BYTES) != cudaSuccess) return ACO_ERR_CUDA;
    head_kernel<<<(unsigned)std::min<size_t>((E + 127) / 128, (size_t)sm_count() * 2), TPB, HeadSmem::BYTES, st>>>(
        E, params, o, w.e + (size_t)layers * E * H, scores, nullptr, 0.f, 0.f, nullptr, nullptr, nullptr, w.status);
    return cudaGetLastError() == cudaSuccess ? ACO_OK : ACO_ERR_CUDA;
}

int aco_mpnn_grad(int n_nodes, int k, int layers, const float *params, const float *node_feat, const float *edge_feat,
                  const int *nbr, const float *labels, float pos_weight, void *workspace, size_t ws_bytes, float *grad,
                  float *loss, float *scores, void *stream)
{
    if (!args_ok(n_nodes, k, layers) || !params || !node_feat || !edge_feat || !nbr || !labels || !workspace ||
        !grad || !loss)
        return ACO_ERR_INVALID;
    const Workspace w = carve(workspace, n_nodes, k, layers);
    if (ws_bytes < w.bytes) return ACO_ERR_CAPACITY;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const ParamOffsets o = param_offsets(layers);
    const size_t E = (size_t)n_nodes * k;
    const int N = n_nodes, L = layers, grid_sm = sm_count() * 2;
    if (cudaMemsetAsync(w.status, 0, 64, st) != cudaSuccess) return ACO_ERR_CUDA;
    if (cudaMemsetAsync(grad, 0, sizeof(float) * o.count, st) != cudaSuccess) return ACO_ERR_CUDA;
    if (cudaMemsetAsync(loss, 0, sizeof(float), st) != cudaSuccess) return ACO_ERR_CUDA;
    if (cudaMemsetAsync(w.dh, 0, sizeof(float) * N * H, st) != cudaSuccess) return ACO_ERR_CUDA;
    int rc = run_forward(N, k, L, params, node_feat, edge_feat, nbr, w, st);
    if (rc != ACO_OK) return rc;
    if (set_smem(head_kernel, HeadSmem::BYTES) != cudaSuccess) return ACO_ERR_CUDA;
    head_kernel<<<(unsigned)std::min<size_t>((E + 127) / 128, (size_t)grid_sm), TPB, HeadSmem::BYTES, st>>>(
        E, params, o, w.e + (size_t)L * E * H, scores ? scores : w.s, labels, pos_weight, 1.0f / (float)E, w.de, grad,
        loss, w.status);
    if (set_smem(edge_bwd_kernel, EdgeBwdSmem::BYTES) != cudaSuccess) return ACO_ERR_CUDA;
    if (set_smem(node_bwd_kernel, NodeBwdSmem::BYTES) != cudaSuccess) return ACO_ERR_CUDA;
    const int ntiles = (N + 127) / 128, npt = 128 / k, etiles = (N + npt - 1) / npt;
    for (int l = L - 1; l >= 0; l--) {
        float *dP = w.dP;
        if (cudaMemsetAsync(dP, 0, sizeof(float) * N * 4 * H, st) != cudaSuccess) return ACO_ERR_CUDA;
        edge_bwd_kernel<<<std::min(etiles, grid_sm), TPB, EdgeBwdSmem::BYTES, st>>>(
            N, k, params + o.A[l], w.P + (size_t)l * N * 4 * H, w.u + (size_t)l * N * H, w.q + (size_t)l * E * H,
            w.e + (size_t)l * E * H, w.e + (size_t)(l + 1) * E * H, nbr, w.dh, w.de, dP, grad + o.A[l], grad + o.a[l],
            w.status);
        node_bwd_kernel<<<std::min(ntiles, grid_sm), TPB, NodeBwdSmem::BYTES, st>>>(
            N, params + o.W[l], w.h + (size_t)l * N * H, dP, w.dh, grad + o.W[l], grad + o.b[l], w.status);
    }
    embed_bwd_kernel<<<H, 256, 0, st>>>(N, k, o, node_feat, edge_feat, w.dh, w.de, grad);
    return cudaGetLastError() == cudaSuccess ? ACO_OK : ACO_ERR_CUDA;
}

int aco_mpnn_adam(int count, float *params, const float *grad, float *m, float *v, float lr, float beta1, float beta2,
                  float eps, int step, void *stream)
{
    if (count <= 0 || !params || !grad || !m || !v || step < 1) return ACO_ERR_INVALID;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<std::min((count + 255) / 256, 1024), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        count, params, grad, m, v, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? ACO_OK : ACO_ERR_CUDA;
}

int aco_mpnn_status(void *workspace, void *stream)
{
    if (!workspace) return ACO_ERR_INVALID;
    int h = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(&h, workspace, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return ACO_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return ACO_ERR_CUDA;
    return h;
}

} // extern "C"
