// peaks.cu -- care-b200-peaks: measured integer-pipe peaks of this GPU for
// the alignment stage's roofline.
//
// The alignment's unit of work is one 32-bit word compare of the shifted
// Hamming distance on bit planes: two funnel shifts (hi and lo plane of the
// candidate window), two XORs with the anchor's planes, an OR, a POPC and an
// add. This program times, in registers only (no memory traffic):
//   popc   -- POPC alone, 8 independent chains per thread;
//   word   -- the full word-compare mix above, 4 independent chains.
// Prints one JSON object: {"popc_per_s": .., "word_compares_per_s": .., ...}.
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
    if (cudaGetLastError() != cudaSuccess) { std::fprintf(stderr, "launch failed\n"); return 1; }
    const double n = (double)blocks * threads * iters;
    std::printf("{\"popc_per_s\": %.6e, \"word_compares_per_s\": %.6e, \"popc_ms\": %.4f, \"word_ms\": %.4f, "
                "\"sms\": %d, \"clock_khz\": %d}\n",
                n * 8 / (tp / 1e3), n * 4 / (tw / 1e3), tp, tw, sms, clk);
    cudaFree(out);
    return 0;
}
