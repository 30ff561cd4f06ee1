// mlp.cu -- the learned decision network (24 -> 64 -> 64 -> 1, GELU) on the
// Blackwell tensor cores: batched inference, training (forward + backward of
// a 128-row tile per step of a persistent CTA), gradient reduction and Adam.
//
// Every GEMM is a tcgen05.mma of kind::f16 (bfloat16 A and B in shared
// memory, FP32 accumulator in tensor memory) issued by one thread; the
// epilogues read the accumulators back with tcgen05.ld, one TMEM lane (= one
// tile row) per thread. Bias gradients come out of the weight-gradient GEMMs
// through a row of ones appended to the B operand.
#include "../../include/care_b200.h"
#include "mlp.hpp"
#include "tc05.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace careb200;
using namespace careb200::tc05;

namespace {

constexpr int NF = 24, KP = 32, H = 64, TILE = 128;
constexpr int OW1 = 0, OB1 = 1536, OW2 = 1600, OB2 = 5696, OW3 = 5760, OB3 = 5824;
constexpr int NPARAM = 5825, OMEAN = 5825, OISTD = 5849, NFLOATS = 5873;
constexpr int PSTRIDE = 5888;          // per-CTA partial: NPARAM gradient values, then the loss sum
constexpr int TRAIN_CTAS = 148;
constexpr int INFER_CTAS_PER_SM = 4;
static_assert(NFLOATS == kMlpFloats && NFLOATS == CARE_B200_MLP_FLOATS && NPARAM == CARE_B200_MLP_PARAMS, "layout");

// inference shared memory: A tiles of the two layers, both weight tiles
constexpr int I_A = 0, I_H = 8192, I_W1 = 24576, I_W2 = 28672, I_BYTES = 36864;
// training shared memory
constexpr int S_X = 0;                 // x       128 x 32  (A of z1)
constexpr int S_XT = 8192;             // x^T|1    32 x 128 (B of gW1|gb1)
constexpr int S_H1 = 16384;            // h1      128 x 64  (A of z2)
constexpr int S_H1T = 32768;           // h1^T|1   80 x 128 (B of gW2|gb2)
constexpr int S_D2 = 53248;            // dz2     128 x 64  (A of dh1)
constexpr int S_DT = 69632;            // dz2^T, then dz1^T: 128 x 128, rows 64.. zero (A of gW2, gW1)
constexpr int S_W1 = 102400;           // W1       64 x 32
constexpr int S_W2 = 106496;           // W2       64 x 64  (row n2, K = n1)
constexpr int S_W2T = 114688;          // W2^T     64 x 64  (row n1, K = n2)
constexpr int S_BYTES = 122880;
// training tensor-memory columns
constexpr int C_Z1 = 0, C_Z2 = 64, C_GW2 = 128, C_GW1 = 224, TRAIN_TMEM = 256;
constexpr int N_GW2 = 80, N_GW1 = 32;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// 8 consecutive K elements of a row (one 16-byte core-matrix row)
__device__ __forceinline__ void st8(uint8_t* tile, int row, int k0, int K, const float* v) {
    *reinterpret_cast<uint4*>(tile + kmajor_off(row, k0, K)) =
        make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}
__device__ __forceinline__ void st1(uint8_t* tile, int row, int k, int K, float v) {
    *reinterpret_cast<__nv_bfloat16*>(tile + kmajor_off(row, k, K)) = __float2bfloat16_rn(v);
}

// GELU with the Gauss error function, and its derivative
__device__ __forceinline__ float gelu(float x) {
    return __fmul_rn(__fmul_rn(0.5f, x), __fadd_rn(1.0f, erff(__fmul_rn(x, 0.70710678118654752f))));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = __fmul_rn(0.5f, __fadd_rn(1.0f, erff(__fmul_rn(x, 0.70710678118654752f))));
    const float pdf = __fmul_rn(expf(__fmul_rn(__fmul_rn(-0.5f, x), x)), 0.39894228040143268f);
    return __fadd_rn(cdf, __fmul_rn(x, pdf));
}

__device__ void stage_weights(const float* __restrict__ P, uint8_t* sW1, uint8_t* sW2, uint8_t* sW2t) {
    for (int i = threadIdx.x; i < H * KP; i += blockDim.x) {
        const int n = i / KP, k = i % KP;
        st1(sW1, n, k, KP, k < NF ? P[OW1 + n * NF + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
        const int n = i / H, k = i % H;
        const float w = P[OW2 + i];
        st1(sW2, n, k, H, w);
        if (sW2t) st1(sW2t, k, n, H, w);
    }
}

// shared-memory operands written by the threads are handed to the tensor
// core, and tensor-memory reads of the threads are ordered before it
__device__ __forceinline__ void operands_ready() {
    fence_smem_to_async();
    fence_before_sync();
    __syncthreads();
}

// D(tmem) (+)= A x B^T over K (a multiple of 16); A and B K-major tiles
__device__ __forceinline__ void issue(uint32_t d, const uint8_t* A, const uint8_t* B, int K, uint32_t idesc,
                                      bool accumulate) {
    const uint32_t a0 = smem_addr(A), b0 = smem_addr(B);
    const uint32_t sbo = (uint32_t)(K / 8) * 128u;
    for (int s = 0; s < K / 16; ++s)
        mma_bf16(d, make_desc(a0 + 256u * s, sbo), make_desc(b0 + 256u * s, sbo), idesc, accumulate || s > 0);
}

// all threads wait for the work committed to `bar`; false in every thread
// when any thread's bounded wait ran out
__device__ __forceinline__ bool wait_all(uint64_t* bar, uint32_t& phase) {
    const bool ok = mbar_wait(bar, phase);
    if (__syncthreads_or(!ok)) return false;
    phase ^= 1u;
    fence_after_sync();
    return true;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}

// ---------------------------------------------------------------------------
// Inference: persistent CTAs of 128 threads, one 128-row tile at a time.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ P, const float* __restrict__ X,
                                                   uint64_t n_host, const unsigned long long* __restrict__ n_dev,
                                                   float* __restrict__ logit, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* sA = sm + I_A;
    uint8_t* sH = sm + I_H;
    uint8_t* sW1 = sm + I_W1;
    uint8_t* sW2 = sm + I_W2;
    __shared__ float s_b1[H], s_b2[H], s_w3[H], s_mean[NF], s_istd[NF];
    __shared__ float s_b3;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint64_t n = n_dev ? min((uint64_t)*n_dev, n_host) : n_host;

    stage_weights(P, sW1, sW2, nullptr);
    if (tid < H) { s_b1[tid] = P[OB1 + tid]; s_b2[tid] = P[OB2 + tid]; s_w3[tid] = bf16r(P[OW3 + tid]); }
    if (tid < NF) { s_mean[tid] = P[OMEAN + tid]; s_istd[tid] = P[OISTD + tid]; }
    if (tid == 0) { s_b3 = P[OB3]; mbar_init(&s_bar, 1); }
    if (warp == 0) tmem_alloc(&s_tmem, 64);
    operands_ready();
    fence_after_sync();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t idesc = idesc_bf16_f32(TILE, H);
    uint32_t phase = 0;
    bool ok = true;
    const uint64_t ntiles = (n + TILE - 1) / TILE;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t row = tile * TILE + tid;
        float xn[KP];
#pragma unroll
        for (int k = 0; k < KP; ++k) xn[k] = 0.0f;
        if (row < n) {
            const float4* src = reinterpret_cast<const float4*>(X + row * NF);
#pragma unroll
            for (int q = 0; q < NF / 4; ++q) {
                const float4 v = __ldg(src + q);
                xn[4 * q] = v.x; xn[4 * q + 1] = v.y; xn[4 * q + 2] = v.z; xn[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int k = 0; k < NF; ++k) xn[k] = bf16r(__fmul_rn(__fsub_rn(xn[k], s_mean[k]), s_istd[k]));
        }
#pragma unroll
        for (int c = 0; c < KP / 8; ++c) st8(sA, tid, 8 * c, KP, xn + 8 * c);
        operands_ready();
        if (tid == 0) { fence_after_sync(); issue(tmem, sA, sW1, KP, idesc, false); commit(&s_bar); }
        if (!(ok = wait_all(&s_bar, phase))) break;
#pragma unroll
        for (int c = 0; c < H / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = bf16r(gelu(__fadd_rn(v[i], s_b1[16 * c + i])));
            st8(sH, tid, 16 * c, H, v);
            st8(sH, tid, 16 * c + 8, H, v + 8);
        }
        operands_ready();
        if (tid == 0) { fence_after_sync(); issue(tmem, sH, sW2, H, idesc, false); commit(&s_bar); }
        if (!(ok = wait_all(&s_bar, phase))) break;
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < H / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) s = __fadd_rn(s, __fmul_rn(bf16r(gelu(__fadd_rn(v[i], s_b2[16 * c + i]))), s_w3[16 * c + i]));
        }
        if (row < n) logit[row] = __fadd_rn(s, s_b3);
    }
    if (!ok) {
        if (tid == 0) atomicOr(err, 1);
        mbar_wait(&s_bar, phase);     // an MMA still in flight finishes before its TMEM is released
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) { fence_after_sync(); tmem_dealloc(tmem, 64); }
}

// ---------------------------------------------------------------------------
// Training: gradient of the mean (optionally row-weighted) binary
// cross-entropy over rows [off, off+cnt) of the (optionally permuted)
// resident data. Each CTA walks
// its tiles and keeps gW2|gb2 and gW1|gb1 accumulating in tensor memory, the
// w3/b3 gradients and the loss in registers; at the end it writes one
// partial per CTA (summed in CTA order by k_mlp_reduce).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ X,
                                                     const float* __restrict__ Y, const float* __restrict__ Wt,
                                                     const uint32_t* __restrict__ perm,
                                                     uint64_t off, uint64_t cnt, float inv_b,
                                                     float* __restrict__ part, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* sX = sm + S_X;
    uint8_t* sXt = sm + S_XT;
    uint8_t* sH1 = sm + S_H1;
    uint8_t* sH1t = sm + S_H1T;
    uint8_t* sD2 = sm + S_D2;
    uint8_t* sDt = sm + S_DT;
    __shared__ float s_b1[H], s_b2[H], s_w3[H], s_mean[NF], s_istd[NF];
    __shared__ float s_b3;
    __shared__ float s_g3[4][H + 2];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    stage_weights(P, sm + S_W1, sm + S_W2, sm + S_W2T);
    // constant operand rows: a row of ones under x^T and h1^T (bias
    // gradients), zeros in the padding rows
    for (int i = tid; i < (KP - NF) * TILE; i += TILE) st1(sXt, NF + i / TILE, i % TILE, TILE, i < TILE ? 1.0f : 0.0f);
    for (int i = tid; i < (N_GW2 - H) * TILE; i += TILE) st1(sH1t, H + i / TILE, i % TILE, TILE, i < TILE ? 1.0f : 0.0f);
    for (int i = tid; i < (TILE - H) * TILE; i += TILE) st1(sDt, H + i / TILE, i % TILE, TILE, 0.0f);
    if (tid < H) { s_b1[tid] = P[OB1 + tid]; s_b2[tid] = P[OB2 + tid]; s_w3[tid] = bf16r(P[OW3 + tid]); }
    if (tid < NF) { s_mean[tid] = P[OMEAN + tid]; s_istd[tid] = P[OISTD + tid]; }
    if (tid == 0) { s_b3 = P[OB3]; mbar_init(&s_bar, 1); }
    if (warp == 0) tmem_alloc(&s_tmem, TRAIN_TMEM);
    operands_ready();
    fence_after_sync();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t id64 = idesc_bf16_f32(TILE, H), id80 = idesc_bf16_f32(TILE, N_GW2), id32 = idesc_bf16_f32(TILE, N_GW1);
    uint32_t phase = 0;
    bool ok = true, first = true;
    float acc_lo = 0.0f, acc_hi = 0.0f, acc_b3 = 0.0f, acc_loss = 0.0f;
    const uint64_t ntiles = (cnt + TILE - 1) / TILE;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t i = tile * TILE + tid;
        const bool valid = i < cnt;
        float xn[KP];
        float y = 0.0f, w = 1.0f;
#pragma unroll
        for (int k = 0; k < KP; ++k) xn[k] = 0.0f;
        if (valid) {
            const uint64_t src = perm ? perm[off + i] : off + i;
            const float4* px = reinterpret_cast<const float4*>(X + src * NF);
#pragma unroll
            for (int q = 0; q < NF / 4; ++q) {
                const float4 v = __ldg(px + q);
                xn[4 * q] = v.x; xn[4 * q + 1] = v.y; xn[4 * q + 2] = v.z; xn[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int k = 0; k < NF; ++k) xn[k] = bf16r(__fmul_rn(__fsub_rn(xn[k], s_mean[k]), s_istd[k]));
            y = Y[src];
            if (Wt) w = Wt[src];
        }
#pragma unroll
        for (int c = 0; c < KP / 8; ++c) st8(sX, tid, 8 * c, KP, xn + 8 * c);
#pragma unroll
        for (int k = 0; k < NF; ++k) st1(sXt, k, tid, TILE, xn[k]);
        // z1 = x W1^T
        operands_ready();
        if (tid == 0) { fence_after_sync(); issue(tmem + C_Z1, sX, sm + S_W1, KP, id64, false); commit(&s_bar); }
        if (!(ok = wait_all(&s_bar, phase))) break;
        // h1 = gelu(z1 + b1); z2 = h1 W2^T
#pragma unroll
        for (int c = 0; c < H / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + C_Z1 + 16 * c, v);
#pragma unroll
            for (int e = 0; e < 16; ++e) v[e] = bf16r(gelu(__fadd_rn(v[e], s_b1[16 * c + e])));
            st8(sH1, tid, 16 * c, H, v);
            st8(sH1, tid, 16 * c + 8, H, v + 8);
#pragma unroll
            for (int e = 0; e < 16; ++e) st1(sH1t, 16 * c + e, tid, TILE, v[e]);
        }
        operands_ready();
        if (tid == 0) { fence_after_sync(); issue(tmem + C_Z2, sH1, sm + S_W2, H, id64, false); commit(&s_bar); }
        if (!(ok = wait_all(&s_bar, phase))) break;
        // logit, loss and dL/dlogit
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < H / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + C_Z2 + 16 * c, v);
#pragma unroll
            for (int e = 0; e < 16; ++e) s = __fadd_rn(s, __fmul_rn(bf16r(gelu(__fadd_rn(v[e], s_b2[16 * c + e]))), s_w3[16 * c + e]));
        }
        const float l = __fadd_rn(s, s_b3);
        const float pr = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-l)));
        const float dl = valid ? __fmul_rn(__fmul_rn(__fsub_rn(pr, y), w), inv_b) : 0.0f;
        const float li = valid ? __fmul_rn(__fadd_rn(__fsub_rn(fmaxf(l, 0.0f), __fmul_rn(l, y)), log1pf(expf(-fabsf(l)))), w) : 0.0f;
        // gradients of w3 (warp sums) and dz2 = dl w3 gelu'(a2)
#pragma unroll
        for (int c = 0; c < H / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + C_Z2 + 16 * c, v);
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int j = 16 * c + e;
                const float a2 = __fadd_rn(v[e], s_b2[j]);
                const float g = warp_sum(__fmul_rn(dl, bf16r(gelu(a2))));
                if (lane == (j & 31)) { if (j < 32) acc_lo = __fadd_rn(acc_lo, g); else acc_hi = __fadd_rn(acc_hi, g); }
                v[e] = bf16r(__fmul_rn(__fmul_rn(dl, s_w3[j]), gelu_grad(a2)));
            }
            st8(sD2, tid, 16 * c, H, v);
            st8(sD2, tid, 16 * c + 8, H, v + 8);
#pragma unroll
            for (int e = 0; e < 16; ++e) st1(sDt, 16 * c + e, tid, TILE, v[e]);
        }
        {
            const float gb = warp_sum(dl), gl = warp_sum(li);
            if (lane == 0) { acc_b3 = __fadd_rn(acc_b3, gb); acc_loss = __fadd_rn(acc_loss, gl); }
        }
        // dh1 = dz2 W2 (over z2's columns); gW2|gb2 += dz2^T [h1 | 1]
        operands_ready();
        if (tid == 0) {
            fence_after_sync();
            issue(tmem + C_Z2, sD2, sm + S_W2T, H, id64, false);
            issue(tmem + C_GW2, sDt, sH1t, TILE, id80, !first);
            commit(&s_bar);
        }
        if (!(ok = wait_all(&s_bar, phase))) break;
        // dz1 = dh1 gelu'(z1 + b1); gW1|gb1 += dz1^T [x | 1]
#pragma unroll
        for (int c = 0; c < H / 16; ++c) {
            float dh[16], z[16];
            tmem_ld16(lane_addr + C_Z2 + 16 * c, dh);
            tmem_ld16(lane_addr + C_Z1 + 16 * c, z);
#pragma unroll
            for (int e = 0; e < 16; ++e)
                st1(sDt, 16 * c + e, tid, TILE, bf16r(__fmul_rn(dh[e], gelu_grad(__fadd_rn(z[e], s_b1[16 * c + e])))));
        }
        operands_ready();
        if (tid == 0) { fence_after_sync(); issue(tmem + C_GW1, sDt, sXt, TILE, id32, !first); commit(&s_bar); }
        if (!(ok = wait_all(&s_bar, phase))) break;
        first = false;
    }
    if (!ok) {
        if (tid == 0) atomicOr(err, 1);
        mbar_wait(&s_bar, phase);
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    float* out = part + (size_t)blockIdx.x * PSTRIDE;
    if (warp < 2) {                       // TMEM lanes 0..63 hold the output rows
        const int nrow = tid;
#pragma unroll
        for (int c = 0; c < N_GW2 / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + C_GW2 + 16 * c, v);
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int col = 16 * c + e;
                const float g = first ? 0.0f : v[e];
                if (col < H) out[OW2 + nrow * H + col] = g;
                else if (col == H) out[OB2 + nrow] = g;
            }
        }
#pragma unroll
        for (int c = 0; c < N_GW1 / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + C_GW1 + 16 * c, v);
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int col = 16 * c + e;
                const float g = first ? 0.0f : v[e];
                if (col < NF) out[OW1 + nrow * NF + col] = g;
                else if (col == NF) out[OB1 + nrow] = g;
            }
        }
    }
    s_g3[warp][lane] = acc_lo;
    s_g3[warp][lane + 32] = acc_hi;
    if (lane == 0) { s_g3[warp][H] = acc_b3; s_g3[warp][H + 1] = acc_loss; }
    fence_before_sync();
    __syncthreads();
    if (tid < H + 2) {
        const float g = __fadd_rn(__fadd_rn(__fadd_rn(s_g3[0][tid], s_g3[1][tid]), s_g3[2][tid]), s_g3[3][tid]);
        out[tid < H ? OW3 + tid : (tid == H ? OB3 : NPARAM)] = g;
    }
    if (warp == 0) { fence_after_sync(); tmem_dealloc(tmem, TRAIN_TMEM); }
}

// Sum of the CTA partials in CTA order; optionally the Adam update
// (bias-corrected moments; bc holds 1-beta1^t, 1-beta2^t per step).
__global__ void k_mlp_reduce(const float* __restrict__ part, int nparts, float* __restrict__ P,
                             float* __restrict__ m, float* __restrict__ v, float* __restrict__ grad,
                             float* __restrict__ loss, float inv_b, int adam, float lr, float b1, float omb1,
                             float b2, float omb2, float eps, const float* __restrict__ bc, int step) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > NPARAM) return;
    float g = 0.0f;
    for (int c = 0; c < nparts; ++c) g = __fadd_rn(g, part[(size_t)c * PSTRIDE + p]);
    if (p == NPARAM) {
        if (loss) loss[step] = __fmul_rn(g, inv_b);
        return;
    }
    if (grad) grad[p] = g;
    if (adam) {
        const float mm = __fadd_rn(__fmul_rn(b1, m[p]), __fmul_rn(omb1, g));
        const float vv = __fadd_rn(__fmul_rn(b2, v[p]), __fmul_rn(__fmul_rn(omb2, g), g));
        m[p] = mm;
        v[p] = vv;
        const float mh = __fdiv_rn(mm, bc[2 * step]), vh = __fdiv_rn(vv, bc[2 * step + 1]);
        P[p] = __fsub_rn(P[p], __fdiv_rn(__fmul_rn(lr, mh), __fadd_rn(__fsqrt_rn(vh), eps)));
    }
}

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// uniform in [-1, 1)
float uniform_pm1(uint64_t& s) { return (float)((double)(splitmix64(s) >> 11) * (2.0 / 9007199254740992.0) - 1.0); }

}  // namespace

namespace careb200 {

cudaError_t mlp_infer(const float* params, const float* x, uint64_t n, const unsigned long long* n_dev,
                      float* logits, int* err, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)sms * INFER_CTAS_PER_SM);
    k_mlp_infer<<<grid, TILE, I_BYTES, stream>>>(params, x, n, n_dev, logits, err);
    return cudaGetLastError();
}

}  // namespace careb200

struct care_b200_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    float* d_p = nullptr;             // NFLOATS
    float* d_m = nullptr;             // Adam moments, NPARAM each
    float* d_v = nullptr;
    float* d_part = nullptr;          // TRAIN_CTAS * PSTRIDE
    float* d_grad = nullptr;          // NPARAM
    int* d_err = nullptr;
    float* d_loss = nullptr;          // per step
    float* d_bc = nullptr;            // 2 per step
    uint64_t step_cap = 0;
    float* d_x = nullptr;             // rows handed in by the caller
    float* d_y = nullptr;             // labels, or logits of care_b200_mlp_forward
    float* d_w = nullptr;             // row weights
    uint64_t xcap = 0, ycap = 0, wcap = 0;
    float* d_tx = nullptr;            // resident training rows
    float* d_ty = nullptr;
    float* d_tw = nullptr;            // null: every row weighs 1
    uint64_t n_train = 0;
    uint32_t* d_perm = nullptr;
    uint64_t perm_cap = 0;
    int64_t t = 0;                    // Adam steps taken
};

namespace {

int mfail(care_b200_mlp* m, int code, const std::string& msg) {
    if (m) m->err = msg;
    return code;
}

#define MCK(call, where)                                                                              \
    do {                                                                                              \
        const cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return mfail(m, CARE_B200_ECUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
cudaError_t grow(T*& p, uint64_t& cap, uint64_t need) {
    if (need <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const cudaError_t e = cudaMalloc(&p, std::max<uint64_t>(need, 1) * sizeof(T));
    if (e == cudaSuccess) cap = need;
    return e;
}

int upload_rows(care_b200_mlp* m, const float* x, const float* y, const float* w, uint64_t n) {
    MCK(grow(m->d_x, m->xcap, n * NF), "alloc rows");
    MCK(grow(m->d_y, m->ycap, n), "alloc labels");
    if (w) {
        MCK(grow(m->d_w, m->wcap, n), "alloc weights");
        MCK(cudaMemcpyAsync(m->d_w, w, n * 4, cudaMemcpyHostToDevice, m->stream), "upload weights");
    }
    MCK(cudaMemcpyAsync(m->d_x, x, n * NF * 4, cudaMemcpyHostToDevice, m->stream), "upload rows");
    if (y) MCK(cudaMemcpyAsync(m->d_y, y, n * 4, cudaMemcpyHostToDevice, m->stream), "upload labels");
    return CARE_B200_OK;
}

int ensure_steps(care_b200_mlp* m, uint64_t steps) {
    if (steps <= m->step_cap) return CARE_B200_OK;
    uint64_t c1 = 0, c2 = 0;
    if (m->d_loss) cudaFree(m->d_loss);
    if (m->d_bc) cudaFree(m->d_bc);
    m->d_loss = nullptr;
    m->d_bc = nullptr;
    m->step_cap = 0;
    MCK(grow(m->d_loss, c1, steps), "alloc losses");
    MCK(grow(m->d_bc, c2, 2 * steps), "alloc bias corrections");
    m->step_cap = steps;
    return CARE_B200_OK;
}

int check_err(care_b200_mlp* m) {
    int e = 0;
    MCK(cudaMemcpyAsync(&e, m->d_err, 4, cudaMemcpyDeviceToHost, m->stream), "error flag");
    MCK(cudaStreamSynchronize(m->stream), "sync");
    if (e) return mfail(m, CARE_B200_ECUDA, "tensor-core completion wait ran out");
    return CARE_B200_OK;
}

// gradient partials of rows [off, off+cnt) and their reduction (+ Adam)
cudaError_t launch_step(care_b200_mlp* m, const float* X, const float* Y, const float* Wt, const uint32_t* perm, uint64_t off,
                        uint64_t cnt, bool adam, const care_b200_mlp_train_options* o, int step, float* grad) {
    const uint64_t tiles = (cnt + TILE - 1) / TILE;
    const int ctas = (int)std::min<uint64_t>(tiles, TRAIN_CTAS);
    const float inv_b = 1.0f / (float)cnt;
    k_mlp_grad<<<ctas, TILE, S_BYTES, m->stream>>>(m->d_p, X, Y, Wt, perm, off, cnt, inv_b, m->d_part, m->d_err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const double b1 = o ? o->beta1 : 0.9, b2 = o ? o->beta2 : 0.999;
    k_mlp_reduce<<<(NPARAM + 1 + 255) / 256, 256, 0, m->stream>>>(
        m->d_part, ctas, m->d_p, m->d_m, m->d_v, grad, m->d_loss, inv_b, adam ? 1 : 0,
        (float)(o ? o->lr : 1e-3), (float)b1, (float)(1.0 - b1), (float)b2, (float)(1.0 - b2),
        (float)(o ? o->eps : 1e-8), m->d_bc, step);
    return cudaGetLastError();
}

int reset_adam(care_b200_mlp* m) {
    MCK(cudaMemsetAsync(m->d_m, 0, NPARAM * 4, m->stream), "reset");
    MCK(cudaMemsetAsync(m->d_v, 0, NPARAM * 4, m->stream), "reset");
    m->t = 0;
    return CARE_B200_OK;
}

}  // namespace

extern "C" {

void care_b200_mlp_default_train_options(care_b200_mlp_train_options* o) {
    if (!o) return;
    o->epochs = 8;
    o->batch = 65536;
    o->lr = 1e-3;
    o->beta1 = 0.9;
    o->beta2 = 0.999;
    o->eps = 1e-8;
    o->seed = 1;
}

static int care_b200_mlp_create_impl(int device, care_b200_mlp** out);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_mlp_create(int device, care_b200_mlp** out) {
    try {
        return care_b200_mlp_create_impl(device, out);
    } catch (const std::exception&) {
        return CARE_B200_ENOMEM;
    }
}

static int care_b200_mlp_create_impl(int device, care_b200_mlp** out) {
    if (!out) return CARE_B200_EINVAL;
    *out = nullptr;
    auto h = std::make_unique<care_b200_mlp>();
    care_b200_mlp* m = h.get();
    int ndev = 0;
    MCK(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return CARE_B200_EINVAL;
    m->device = device;
    MCK(cudaSetDevice(device), "cudaSetDevice");
    MCK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "stream");
    MCK(cudaMalloc(&m->d_p, NFLOATS * 4), "alloc");
    MCK(cudaMalloc(&m->d_m, NPARAM * 4), "alloc");
    MCK(cudaMalloc(&m->d_v, NPARAM * 4), "alloc");
    MCK(cudaMalloc(&m->d_part, (size_t)TRAIN_CTAS * PSTRIDE * 4), "alloc");
    MCK(cudaMalloc(&m->d_grad, NPARAM * 4), "alloc");
    MCK(cudaMalloc(&m->d_err, 4), "alloc");
    MCK(cudaMemsetAsync(m->d_err, 0, 4, m->stream), "memset");
    MCK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, S_BYTES), "smem attr");
    if (int r = ensure_steps(m, 1)) return r;
    std::vector<float> p(NFLOATS, 0.0f);
    for (int k = 0; k < NF; ++k) p[OISTD + k] = 1.0f;
    MCK(cudaMemcpyAsync(m->d_p, p.data(), NFLOATS * 4, cudaMemcpyHostToDevice, m->stream), "params");
    if (int r = reset_adam(m)) return r;
    MCK(cudaStreamSynchronize(m->stream), "sync");
    *out = h.release();
    return care_b200_mlp_init(*out, 1);
}

int care_b200_mlp_destroy(care_b200_mlp* m) {
    if (!m) return CARE_B200_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (void* p : {(void*)m->d_p, (void*)m->d_m, (void*)m->d_v, (void*)m->d_part, (void*)m->d_grad,
                    (void*)m->d_err, (void*)m->d_loss, (void*)m->d_bc, (void*)m->d_x, (void*)m->d_y,
                    (void*)m->d_tx, (void*)m->d_ty, (void*)m->d_tw, (void*)m->d_perm, (void*)m->d_w})
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return CARE_B200_OK;
}

const char* care_b200_mlp_last_error(const care_b200_mlp* m) { return m ? m->err.c_str() : "no handle"; }

int care_b200_mlp_set_params(care_b200_mlp* m, const float* params) {
    if (!m || !params) return CARE_B200_EINVAL;
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    MCK(cudaMemcpyAsync(m->d_p, params, NFLOATS * 4, cudaMemcpyHostToDevice, m->stream), "params");
    if (int r = reset_adam(m)) return r;
    MCK(cudaStreamSynchronize(m->stream), "sync");
    return CARE_B200_OK;
}

int care_b200_mlp_get_params(care_b200_mlp* m, float* params) {
    if (!m || !params) return CARE_B200_EINVAL;
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    MCK(cudaMemcpyAsync(params, m->d_p, NFLOATS * 4, cudaMemcpyDeviceToHost, m->stream), "params");
    MCK(cudaStreamSynchronize(m->stream), "sync");
    return CARE_B200_OK;
}

int care_b200_mlp_init(care_b200_mlp* m, uint64_t seed) {
    if (!m) return CARE_B200_EINVAL;
    std::vector<float> p(NFLOATS);
    if (int r = care_b200_mlp_get_params(m, p.data())) return r;
    uint64_t s = seed;
    const float a1 = 1.0f / std::sqrt((float)NF), a2 = 1.0f / std::sqrt((float)H);
    for (int i = 0; i < H * NF; ++i) p[OW1 + i] = a1 * uniform_pm1(s);
    for (int i = 0; i < H; ++i) p[OB1 + i] = 0.1f * uniform_pm1(s);
    for (int i = 0; i < H * H; ++i) p[OW2 + i] = a2 * uniform_pm1(s);
    for (int i = 0; i < H; ++i) p[OB2 + i] = 0.1f * uniform_pm1(s);
    for (int i = 0; i < H; ++i) p[OW3 + i] = a2 * uniform_pm1(s);
    p[OB3] = 0.0f;
    return care_b200_mlp_set_params(m, p.data());
}

static int care_b200_mlp_set_data_impl(care_b200_mlp* m, const float* x, const float* labels, const float* weights, uint64_t n,
                           int set_norm);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_mlp_set_data(care_b200_mlp* m, const float* x, const float* labels, const float* weights, uint64_t n,
                           int set_norm) {
    try {
        return care_b200_mlp_set_data_impl(m, x, labels, weights, n, set_norm);
    } catch (const std::exception& e) {
        return m ? mfail(m, CARE_B200_ENOMEM, std::string("care_b200_mlp_set_data: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_mlp_set_data_impl(care_b200_mlp* m, const float* x, const float* labels, const float* weights, uint64_t n,
                           int set_norm) {
    if (!m || !x || !labels || n == 0) return CARE_B200_EINVAL;
    if (n > 0xFFFFFFFFull) return mfail(m, CARE_B200_ELIMIT, "more than 2^32 rows");
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    if (m->d_tx) cudaFree(m->d_tx);
    if (m->d_ty) cudaFree(m->d_ty);
    if (m->d_tw) cudaFree(m->d_tw);
    m->d_tx = m->d_ty = m->d_tw = nullptr;
    m->n_train = 0;
    MCK(cudaMalloc(&m->d_tx, n * NF * 4), "alloc training rows");
    MCK(cudaMalloc(&m->d_ty, n * 4), "alloc training labels");
    MCK(cudaMemcpyAsync(m->d_tx, x, n * NF * 4, cudaMemcpyHostToDevice, m->stream), "upload");
    MCK(cudaMemcpyAsync(m->d_ty, labels, n * 4, cudaMemcpyHostToDevice, m->stream), "upload");
    if (weights) {
        for (uint64_t i = 0; i < n; ++i)
            if (!(weights[i] >= 0.0f) || !std::isfinite(weights[i])) return mfail(m, CARE_B200_EINVAL, "row weights must be finite and >= 0");
        MCK(cudaMalloc(&m->d_tw, n * 4), "alloc training weights");
        MCK(cudaMemcpyAsync(m->d_tw, weights, n * 4, cudaMemcpyHostToDevice, m->stream), "upload");
    }
    m->n_train = n;
    if (set_norm) {
        std::vector<double> mu(NF, 0.0), sq(NF, 0.0);
        for (uint64_t i = 0; i < n; ++i)
            for (int k = 0; k < NF; ++k) mu[k] += x[i * NF + k];
        for (int k = 0; k < NF; ++k) mu[k] /= (double)n;
        for (uint64_t i = 0; i < n; ++i)
            for (int k = 0; k < NF; ++k) { const double d = x[i * NF + k] - mu[k]; sq[k] += d * d; }
        std::vector<float> p(NFLOATS);
        MCK(cudaMemcpyAsync(p.data(), m->d_p, NFLOATS * 4, cudaMemcpyDeviceToHost, m->stream), "params");
        MCK(cudaStreamSynchronize(m->stream), "sync");
        for (int k = 0; k < NF; ++k) {
            p[OMEAN + k] = (float)mu[k];
            p[OISTD + k] = (float)(1.0 / std::max(std::sqrt(sq[k] / (double)n), 1e-6));
        }
        MCK(cudaMemcpyAsync(m->d_p, p.data(), NFLOATS * 4, cudaMemcpyHostToDevice, m->stream), "params");
    }
    MCK(cudaStreamSynchronize(m->stream), "sync");
    return CARE_B200_OK;
}

static int care_b200_mlp_gradient_impl(care_b200_mlp* m, const float* x, const float* labels, const float* weights, uint64_t n,
                           float* grad, float* loss);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_mlp_gradient(care_b200_mlp* m, const float* x, const float* labels, const float* weights, uint64_t n,
                           float* grad, float* loss) {
    try {
        return care_b200_mlp_gradient_impl(m, x, labels, weights, n, grad, loss);
    } catch (const std::exception& e) {
        return m ? mfail(m, CARE_B200_ENOMEM, std::string("care_b200_mlp_gradient: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_mlp_gradient_impl(care_b200_mlp* m, const float* x, const float* labels, const float* weights, uint64_t n,
                           float* grad, float* loss) {
    if (!m || !x || !labels || n == 0 || !grad) return CARE_B200_EINVAL;
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    if (int r = upload_rows(m, x, labels, weights, n)) return r;
    MCK(launch_step(m, m->d_x, m->d_y, weights ? m->d_w : nullptr, nullptr, 0, n, false, nullptr, 0, m->d_grad),
        "k_mlp_grad");
    MCK(cudaMemcpyAsync(grad, m->d_grad, NPARAM * 4, cudaMemcpyDeviceToHost, m->stream), "gradient");
    float l = 0.0f;
    MCK(cudaMemcpyAsync(&l, m->d_loss, 4, cudaMemcpyDeviceToHost, m->stream), "loss");
    if (int r = check_err(m)) return r;
    if (loss) *loss = l;
    return CARE_B200_OK;
}

static int care_b200_mlp_train_step_impl(care_b200_mlp* m, const float* x, const float* labels, const float* weights,
                             uint64_t n, const care_b200_mlp_train_options* o, float* loss);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_mlp_train_step(care_b200_mlp* m, const float* x, const float* labels, const float* weights,
                             uint64_t n, const care_b200_mlp_train_options* o, float* loss) {
    try {
        return care_b200_mlp_train_step_impl(m, x, labels, weights, n, o, loss);
    } catch (const std::exception& e) {
        return m ? mfail(m, CARE_B200_ENOMEM, std::string("care_b200_mlp_train_step: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_mlp_train_step_impl(care_b200_mlp* m, const float* x, const float* labels, const float* weights,
                             uint64_t n, const care_b200_mlp_train_options* o, float* loss) {
    if (!m || !x || !labels || n == 0 || !o) return CARE_B200_EINVAL;
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    if (int r = upload_rows(m, x, labels, weights, n)) return r;
    const int64_t t = m->t + 1;
    const float bc[2] = {(float)(1.0 - std::pow(o->beta1, (double)t)), (float)(1.0 - std::pow(o->beta2, (double)t))};
    MCK(cudaMemcpyAsync(m->d_bc, bc, 8, cudaMemcpyHostToDevice, m->stream), "bias corrections");
    MCK(launch_step(m, m->d_x, m->d_y, weights ? m->d_w : nullptr, nullptr, 0, n, true, o, 0, nullptr), "k_mlp_grad");
    float l = 0.0f;
    MCK(cudaMemcpyAsync(&l, m->d_loss, 4, cudaMemcpyDeviceToHost, m->stream), "loss");
    if (int r = check_err(m)) return r;
    m->t = t;
    if (loss) *loss = l;
    return CARE_B200_OK;
}

static int care_b200_mlp_train_impl(care_b200_mlp* m, const care_b200_mlp_train_options* o, float* losses,
                        uint64_t loss_capacity, uint64_t* num_steps);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_mlp_train(care_b200_mlp* m, const care_b200_mlp_train_options* o, float* losses,
                        uint64_t loss_capacity, uint64_t* num_steps) {
    try {
        return care_b200_mlp_train_impl(m, o, losses, loss_capacity, num_steps);
    } catch (const std::exception& e) {
        return m ? mfail(m, CARE_B200_ENOMEM, std::string("care_b200_mlp_train: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_mlp_train_impl(care_b200_mlp* m, const care_b200_mlp_train_options* o, float* losses,
                        uint64_t loss_capacity, uint64_t* num_steps) {
    if (!m || !o || o->epochs < 1 || o->batch < 1) return CARE_B200_EINVAL;
    if (m->n_train == 0) return mfail(m, CARE_B200_ESTATE, "no training rows");
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    const uint64_t n = m->n_train, B = (uint64_t)o->batch;
    const uint64_t spe = (n + B - 1) / B, steps = spe * (uint64_t)o->epochs;
    if (int r = ensure_steps(m, steps)) return r;
    // one shuffle per epoch (Fisher-Yates, seeded), all resident for the graph
    MCK(grow(m->d_perm, m->perm_cap, n * (uint64_t)o->epochs), "alloc permutations");
    std::vector<uint32_t> perm(n);
    for (int e = 0; e < o->epochs; ++e) {
        for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
        uint64_t s = o->seed * 0x100000001b3ULL + (uint64_t)e;
        for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix64(s) % (i + 1)]);
        MCK(cudaMemcpy(m->d_perm + (size_t)e * n, perm.data(), n * 4, cudaMemcpyHostToDevice), "upload permutation");
    }
    std::vector<float> bc(2 * steps);
    for (uint64_t k = 0; k < steps; ++k) {
        const double t = (double)(m->t + (int64_t)k + 1);
        bc[2 * k] = (float)(1.0 - std::pow(o->beta1, t));
        bc[2 * k + 1] = (float)(1.0 - std::pow(o->beta2, t));
    }
    MCK(cudaMemcpy(m->d_bc, bc.data(), 8 * steps, cudaMemcpyHostToDevice), "bias corrections");
    // the whole run as one graph: per step the gradient tiles and the update
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    MCK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal), "capture");
    cudaError_t ce = cudaSuccess;
    for (int e = 0; e < o->epochs && ce == cudaSuccess; ++e)
        for (uint64_t k = 0; k < spe && ce == cudaSuccess; ++k) {
            const uint64_t off = k * B, cnt = std::min(B, n - off);
            ce = launch_step(m, m->d_tx, m->d_ty, m->d_tw, m->d_perm + (size_t)e * n, off, cnt, true, o,
                             (int)((uint64_t)e * spe + k), nullptr);
        }
    const cudaError_t ee = cudaStreamEndCapture(m->stream, &graph);
    MCK(ce, "capture launches");
    MCK(ee, "end capture");
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, m->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(m->stream);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    MCK(ce, "training graph");
    if (int r = check_err(m)) return r;
    m->t += (int64_t)steps;
    if (losses && loss_capacity)
        MCK(cudaMemcpy(losses, m->d_loss, std::min(loss_capacity, steps) * 4, cudaMemcpyDeviceToHost), "losses");
    if (num_steps) *num_steps = steps;
    return CARE_B200_OK;
}

static int care_b200_mlp_forward_impl(care_b200_mlp* m, const float* x, uint64_t n, float* logits);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_mlp_forward(care_b200_mlp* m, const float* x, uint64_t n, float* logits) {
    try {
        return care_b200_mlp_forward_impl(m, x, n, logits);
    } catch (const std::exception& e) {
        return m ? mfail(m, CARE_B200_ENOMEM, std::string("care_b200_mlp_forward: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_mlp_forward_impl(care_b200_mlp* m, const float* x, uint64_t n, float* logits) {
    if (!m || !x || !logits) return CARE_B200_EINVAL;
    if (n == 0) return CARE_B200_OK;
    MCK(cudaSetDevice(m->device), "cudaSetDevice");
    if (int r = upload_rows(m, x, nullptr, nullptr, n)) return r;
    // logits land in the label buffer (n floats)
    MCK(mlp_infer(m->d_p, m->d_x, n, nullptr, m->d_y, m->d_err, m->stream), "k_mlp_infer");
    MCK(cudaMemcpyAsync(logits, m->d_y, n * 4, cudaMemcpyDeviceToHost, m->stream), "logits");
    return check_err(m);
}

}  // extern "C"
