// peaks.cu -- care-b200-peaks: measured integer-pipe peaks of this GPU for
// the alignment stage's roofline.
//
// The alignment's unit of work is one 32-bit word compare of the shifted
// Hamming distance on bit planes: two funnel shifts (hi and lo plane of the
// candidate window), two XORs with the anchor's planes, an OR, a POPC and an
// add. This program times, in registers only (no memory traffic):
//   popc   -- POPC alone, 8 independent chains per thread;
//   word   -- the full word-compare mix above, 4 independent chains.
//   msa    -- the MSA stage's per-element update mix (k_peak_msa).
// Prints one JSON object: {"popc_per_s": .., "word_compares_per_s": ..,
// "msa_elements_per_s": .., ...}.
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

__global__ void k_peak_popc(uint32_t seed, int iters, uint32_t* out) {
    uint32_t v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = seed * (threadIdx.x + 1 + j) + blockIdx.x;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = __popc(v[j] ^ (0x9e3779b9u + (uint32_t)i)) + v[j];
    }
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
    if (s == 0x12345678u) out[0] = s;              // keeps the chains live
}

__global__ void k_peak_word(uint32_t seed, int iters, uint32_t* out) {
    uint32_t c[4][4], acc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        acc[j] = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) c[j][k] = seed * (threadIdx.x + 3 * j + k + 1) ^ blockIdx.x;
    }
    const uint32_t ahi = seed ^ 0x85ebca6bu, alo = seed ^ 0xc2b2ae35u;
    for (int i = 0; i < iters; ++i) {
        const uint32_t sh = (uint32_t)i & 31u;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t h = __funnelshift_l(c[j][1], c[j][0], sh);
            const uint32_t l = __funnelshift_l(c[j][3], c[j][2], sh);
            acc[j] += __popc((h ^ ahi) | (l ^ alo));
            c[j][0] ^= acc[j];                      // the next window depends on this one
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) s += acc[j];
    if (s == 0x12345678u) out[0] = s;
}

// The MSA stage's unit of work: one element of a staged candidate row added
// to its column: base and quality code from packed words, weight = factor *
// table[code], four selected adds and a 16-bit count. 4 columns per thread
// (independent chains), registers only.
__global__ void k_peak_msa(uint32_t seed, int iters, uint32_t* out) {
    float wa[4], wc[4], wg[4], wt[4];
    uint32_t cac[4], cgt[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) { wa[j] = wc[j] = wg[j] = wt[j] = 0.0f; cac[j] = cgt[j] = 0u; }
    const float tab[4] = {0.25f, 0.5f, 0.75f, 1.0f};
    uint32_t sw = seed * (threadIdx.x + 1), qw = seed ^ (blockIdx.x * 2654435761u);
    const float fk = 0.9f + 1e-7f * (float)(threadIdx.x & 7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int p = (i + 5 * j) & 15;
            const uint32_t b = (sw >> (30 - 2 * p)) & 3u;
            const uint32_t c = (qw >> (30 - 2 * p)) & 3u;
            const float w = __fmul_rn(fk, c == 0 ? tab[0] : c == 1 ? tab[1] : c == 2 ? tab[2] : tab[3]);
            const uint32_t inc = 1u << (16 * (b & 1u));
            cac[j] += (b & 2u) ? 0u : inc;
            cgt[j] += (b & 2u) ? inc : 0u;
            wa[j] = __fadd_rn(wa[j], b == 0 ? w : 0.0f);
            wc[j] = __fadd_rn(wc[j], b == 1 ? w : 0.0f);
            wg[j] = __fadd_rn(wg[j], b == 2 ? w : 0.0f);
            wt[j] = __fadd_rn(wt[j], b == 3 ? w : 0.0f);
        }
        sw = sw * 1664525u + 1013904223u;            // the next candidate's words
        qw ^= sw;
    }
    float s = 0.0f;
    uint32_t t = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) { s += wa[j] + wc[j] + wg[j] + wt[j]; t += cac[j] + cgt[j]; }
    if (s == 1234.5f && t == 7u) out[0] = t;          // keeps the chains live
}

int main() {
    int dev = 0, sms = 0, clk = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
    uint32_t* out = nullptr;
    if (cudaMalloc(&out, 4) != cudaSuccess) { std::fprintf(stderr, "no device\n"); return 1; }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int threads = 256, blocks = sms * 8, iters = 1 << 14;
    auto run = [&](bool word) {
        float best = 1e30f;
        for (int rep = 0; rep < 5; ++rep) {
            cudaEventRecord(a);
            if (word) k_peak_word<<<blocks, threads>>>(0x1234567u + rep, iters, out);
            else k_peak_popc<<<blocks, threads>>>(0x1234567u + rep, iters, out);
            cudaEventRecord(b);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0 && ms < best) best = ms;     // first launch warms up
        }
        return best;
    };
    const float tp = run(false), tw = run(true);
    float tm = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a);
        k_peak_msa<<<blocks, threads>>>(0x9e3779b9u + rep, iters, out);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && ms < tm) tm = ms;
    }
    if (cudaGetLastError() != cudaSuccess) { std::fprintf(stderr, "launch failed\n"); return 1; }
    const double n = (double)blocks * threads * iters;
    std::printf("{\"popc_per_s\": %.6e, \"word_compares_per_s\": %.6e, \"msa_elements_per_s\": %.6e, "
                "\"popc_ms\": %.4f, \"word_ms\": %.4f, \"msa_ms\": %.4f, \"sms\": %d, \"clock_khz\": %d}\n",
                n * 8 / (tp / 1e3), n * 4 / (tw / 1e3), n * 4 / (tm / 1e3), tp, tw, tm, sms, clk);
    cudaFree(out);
    return 0;
}
