// device.cuh -- shared types and device helpers of the sm_100a correction path.
//
// Sequences: 2-bit codes A=0,C=1,G=2,T=3 packed 16 per uint32, MSB-first
// (the reference's layout, include/sequencehelpers.hpp:152-187). The aligner
// works on "hi/lo bit planes" held in 64-bit words: plane bit i (MSB-first)
// is the high / low bit of base i (the HiLo layout of
// sequencehelpers.hpp:645-697, widened from 32- to 64-bit words).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace careb200 {

constexpr int kMaxLen = 256;          // longest read the kernels accept
constexpr int kMaxMaps = 48;          // maximum_number_of_maps, include/config.hpp:31
constexpr int kPlaneWords = 4;        // 64-bit words per bit plane (kMaxLen / 64)

// Per-launch view of the options (include/options.hpp:36-98).
struct DevOptions {
    int k;
    int num_maps;
    int min_overlap;
    int new_columns;
    int use_quality;
    int quality_bits;
    int exclude_ambiguous;
    int correct_candidates;
    int paired_end;
    int threshold;                    // resultsPerMapThreshold
    int coverage_int;                 // int(estimatedCoverage), the refinement's dataset_coverage
    int correction_type;
    float max_error_rate;
    float min_overlap_ratio;
    float estimated_errorrate;
    float estimated_coverage;
    float m_coverage;
    float paired_filter_threshold;
    unsigned long long kmer_mask;
};

// Device-resident read storage (the CpuReadStorage handle).
struct DevReads {
    const uint32_t* seq;              // n * seq_pitch
    const uint32_t* qual;             // n * qual_pitch or null
    const int32_t* len;
    const uint8_t* ambig;
    int seq_pitch;
    int qual_pitch;
    int max_len;                      // sequenceLengthUpperBound: the quality pitch in chars
    uint32_t n;
};

// One open-addressing slot of a minhash table: key -> [offset, offset+count)
// of that table's value array. count == 0 marks an empty slot.
struct Slot {
    unsigned long long key;
    uint32_t offset;
    uint32_t count;
};

struct TableDesc {
    unsigned long long slot_base;     // index of the table's first slot
    unsigned long long value_base;    // index of the table's first value
    uint32_t mask;                    // capacity - 1 (capacity is a power of two)
    uint32_t pad;
};

// Alignment outcome of one (anchor, candidate) pair, 8 bytes.
struct AlignRes {
    int16_t shift;
    int16_t overlap;
    int16_t nops;
    uint8_t orient;                   // 1 forward, 2 reverse complement, 3 none
    uint8_t paired;                   // PE: mate of the candidate is a candidate of the anchor's mate
};

// A candidate that survived the alignment filters.
struct CandRec {
    uint32_t id;
    int16_t shift;
    uint16_t len;
    float weight;                     // calculateOverlapWeight
    uint32_t orient;                  // 1 forward, 2 reverse complement
};

// Status word written by the kernels.
enum : int {
    kStatusOk = 0,
    kStatusCandOverflow = 1,          // candidate arena too small, rerun with more space
    kStatusCorrOverflow = 2,          // candidate-correction arena too small
    kStatusColumns = 4,               // more MSA columns than the kernel holds
};

// MurmurHash3 64-bit finalizer (the published fmix64), as used by the
// reference's minhasher (hpc_helpers hashers.cuh:85-139).
__device__ __forceinline__ unsigned long long murmur64(unsigned long long x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// Reverse complement of a 32-base 2-bit word (reverse the 2-bit groups,
// complement each code).
__device__ __forceinline__ unsigned long long revcomp64(unsigned long long n) {
    n = ((n >> 2) & 0x3333333333333333ull) | ((n & 0x3333333333333333ull) << 2);
    n = ((n >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((n & 0x0F0F0F0F0F0F0F0Full) << 4);
    n = ((n >> 8) & 0x00FF00FF00FF00FFull) | ((n & 0x00FF00FF00FF00FFull) << 8);
    n = ((n >> 16) & 0x0000FFFF0000FFFFull) | ((n & 0x0000FFFF0000FFFFull) << 16);
    n = (n >> 32) | (n << 32);
    return ~n;
}

// k-mer of k bases starting at base pos of a packed sequence (k <= 32).
__device__ __forceinline__ unsigned long long kmer_at(const uint32_t* s, int k, int pos) {
    const int w = pos >> 4, o = pos & 15;
    // up to three 32-bit words cover 32 bases at any offset
    const unsigned long long hi = ((unsigned long long)s[w] << 32) | (unsigned long long)s[w + 1];
    const unsigned long long lo = (unsigned long long)s[w + 2];
    // 96-bit window [hi:64 | lo:32]; take 2k bits starting at bit 2*o from the top
    const unsigned long long top = o ? (hi << (2 * o)) | (lo >> (32 - 2 * o)) : hi;
    return top >> (64 - 2 * k);
}

// 2-bit code of base p of a packed row.
__device__ __forceinline__ uint32_t base_at(const uint32_t* s, int p) {
    return (s[p >> 4] >> (30 - 2 * (p & 15))) & 3u;
}

// Compress the even bits (0,2,...,30) of x into the low 16 bits, order kept.
__device__ __forceinline__ uint32_t even_bits(uint32_t x) {
    x &= 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    x = (x | (x >> 8)) & 0x0000FFFFu;
    return x;
}

// The 2-bit row of a read -> hi/lo planes of W 64-bit words (+1 zero word).
template <int W>
__device__ __forceinline__ void load_planes(const uint32_t* __restrict__ s, int L,
                                            unsigned long long (&hi)[W + 1],
                                            unsigned long long (&lo)[W + 1]) {
    const int nints = (L + 15) >> 4;
#pragma unroll
    for (int w = 0; w <= W; ++w) { hi[w] = 0; lo[w] = 0; }
#pragma unroll
    for (int w = 0; w < W; ++w) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = 4 * w + q;
            if (idx < nints) {
                const uint32_t x = __ldg(s + idx);
                hi[w] |= (unsigned long long)even_bits(x >> 1) << (48 - 16 * q);
                lo[w] |= (unsigned long long)even_bits(x) << (48 - 16 * q);
            }
        }
        const int valid = L - 64 * w;
        if (valid <= 0) { hi[w] = 0; lo[w] = 0; }
        else if (valid < 64) {
            const unsigned long long m = ~(~0ull >> valid);
            hi[w] &= m; lo[w] &= m;
        }
    }
}

// Planes of the reverse complement of a read of length L given its planes.
template <int W>
__device__ __forceinline__ void revcomp_planes(const unsigned long long (&hi)[W + 1],
                                               const unsigned long long (&lo)[W + 1], int L,
                                               unsigned long long (&rhi)[W + 1],
                                               unsigned long long (&rlo)[W + 1]) {
    // reverse the 64W-bit string word by word
#pragma unroll
    for (int j = 0; j < W; ++j) { rhi[j] = __brevll(hi[W - 1 - j]); rlo[j] = __brevll(lo[W - 1 - j]); }
    rhi[W] = 0; rlo[W] = 0;
    // drop the 64W-L leading bits that came from the padding
    const int d = 64 * W - L;
    const int dq = d >> 6, dr = d & 63;
#pragma unroll
    for (int step = 0; step < W; ++step) {
        if (step < dq) {
#pragma unroll
            for (int j = 0; j < W; ++j) { rhi[j] = rhi[j + 1]; rlo[j] = rlo[j + 1]; }
            rhi[W] = 0; rlo[W] = 0;
        }
    }
    if (dr) {
#pragma unroll
        for (int j = 0; j < W; ++j) {
            rhi[j] = (rhi[j] << dr) | (rhi[j + 1] >> (64 - dr));
            rlo[j] = (rlo[j] << dr) | (rlo[j + 1] >> (64 - dr));
        }
    }
    // complement the L valid bases, keep zeros beyond
#pragma unroll
    for (int j = 0; j < W; ++j) {
        const int valid = L - 64 * j;
        unsigned long long m = valid >= 64 ? ~0ull : (valid <= 0 ? 0ull : ~(~0ull >> valid));
        rhi[j] = (~rhi[j]) & m;
        rlo[j] = (~rlo[j]) & m;
    }
}

struct ShdResult {
    int score, overlap, shift, nops, valid;
};

// One scan direction of the shifted Hamming distance. The "shifted" planes S
// are slid by t = t0..t1 bases against the "other" planes O, exactly in the
// reference's order with its pruning (src/cpu_alignment.cpp:247-316):
// max_errors_excl = min(int(ov*maxErrorRate), best - total + 2*ov); a shift
// with max_errors_excl <= 0 ends the direction; mismatches < max_errors_excl
// and score < best replaces the best (first best kept).
template <int W>
__device__ __forceinline__ void shd_scan(unsigned long long (&Shi)[W + 1], unsigned long long (&Slo)[W + 1],
                                         const unsigned long long (&Ohi)[W + 1],
                                         const unsigned long long (&Olo)[W + 1], int t0, int t1,
                                         int sign, int La, int Lc, int total, float mer, int& best,
                                         int& bestShift) {
    if (t1 < t0) return;
    bool stop = false;
#pragma unroll 1
    for (int q = 0; q <= (t1 >> 6) && !stop; ++q) {
        const int rb = (q == (t0 >> 6)) ? (t0 & 63) : 0;
        const int re = (q == (t1 >> 6)) ? (t1 & 63) : 63;
        if (q >= (t0 >> 6)) {
#pragma unroll 1
            for (int rr = rb; rr <= re; ++rr) {
                const int t = 64 * q + rr;
                const int ov = sign > 0 ? min(La - t, Lc) : min(La, Lc - t);
                int mex = __float2int_rz(__fmul_rn((float)ov, mer));
                mex = min(mex, best - total + 2 * ov);
                if (mex <= 0) { stop = true; break; }
                const int nw = (ov + 63) >> 6;
                int mm = 0;
#pragma unroll
                for (int j = 0; j < W; ++j) {
                    if (j < nw && mm < mex) {
                        const unsigned long long xh = rr ? (Shi[j] << rr) | (Shi[j + 1] >> (64 - rr)) : Shi[j];
                        const unsigned long long xl = rr ? (Slo[j] << rr) | (Slo[j + 1] >> (64 - rr)) : Slo[j];
                        unsigned long long dbits = (xh ^ Ohi[j]) | (xl ^ Olo[j]);
                        const int valid = ov - 64 * j;
                        if (valid < 64) dbits &= ~(~0ull >> valid);
                        mm += __popcll(dbits);
                    }
                }
                if (mm < mex) {
                    const int sc = mm + total - 2 * ov;
                    if (sc < best) { best = sc; bestShift = sign * t; }
                }
            }
        }
        // slide the shifted planes by one 64-base word
#pragma unroll
        for (int j = 0; j < W; ++j) { Shi[j] = Shi[j + 1]; Slo[j] = Slo[j + 1]; }
        Shi[W] = 0; Slo[W] = 0;
    }
}

// cpuShiftedHammingDistancePopcount2BitHiLo (src/cpu_alignment.cpp:32-323).
template <int W>
__device__ __forceinline__ ShdResult shifted_hamming(const unsigned long long (&Ahi)[W + 1],
                                                     const unsigned long long (&Alo)[W + 1], int La,
                                                     const unsigned long long (&Chi)[W + 1],
                                                     const unsigned long long (&Clo)[W + 1], int Lc,
                                                     int minov, float mer) {
    const int total = La + Lc;
    int best = total, bestShift = -Lc;
    unsigned long long Shi[W + 1], Slo[W + 1];
#pragma unroll
    for (int j = 0; j <= W; ++j) { Shi[j] = Ahi[j]; Slo[j] = Alo[j]; }
    shd_scan<W>(Shi, Slo, Chi, Clo, 0, La - minov, +1, La, Lc, total, mer, best, bestShift);
#pragma unroll
    for (int j = 0; j <= W; ++j) { Shi[j] = Chi[j]; Slo[j] = Clo[j]; }
    shd_scan<W>(Shi, Slo, Ahi, Alo, 1, Lc - minov, -1, La, Lc, total, mer, best, bestShift);
    ShdResult r;
    r.valid = bestShift != -Lc;
    const int cb = max(-bestShift, 0);
    const int ce = min(Lc, La - bestShift);
    r.overlap = ce - cb;
    r.score = best;
    r.shift = bestShift;
    r.nops = best - total + 2 * r.overlap;
    return r;
}

// chooseBestAlignmentOrientation (include/alignmentorientation.hpp:12-92).
__device__ __forceinline__ int choose_orientation(const ShdResult& f, const ShdResult& r, int La,
                                                  float min_overlap_ratio, int min_overlap,
                                                  float maxErrorRate) {
    int ret = 3;
    const int lo = __float2int_rz(__fmul_rn((float)La, min_overlap_ratio));
    const int mo = lo > min_overlap ? lo : min_overlap;
    if (f.valid && f.overlap >= mo) {
        if (r.valid && r.overlap >= mo) {
            const float ratio = __fdiv_rn((float)f.nops, (float)f.overlap);
            const float rratio = __fdiv_rn((float)r.nops, (float)r.overlap);
            if (ratio < rratio) { if (ratio < maxErrorRate) ret = 1; }
            else if (rratio < ratio) { if (rratio < maxErrorRate) ret = 2; }
            else if (ratio < maxErrorRate) ret = f.overlap > r.overlap ? 1 : 2;
        } else if (__fdiv_rn((float)f.nops, (float)f.overlap) < maxErrorRate) ret = 1;
    } else if (r.valid && r.overlap >= mo) {
        if (__fdiv_rn((float)r.nops, (float)r.overlap) < maxErrorRate) ret = 2;
    }
    return ret;
}

// feq / fleq / fgeq (include/hostdevicefunctions.cuh:9-29).
__device__ __forceinline__ bool feq(float l, float r) {
    const float d = __fsub_rn(l, r);
    return (d < 0 ? -d : d) < 1e-5f;
}
__device__ __forceinline__ bool fleq(float l, float r) { return (l < r) || feq(l, r); }
__device__ __forceinline__ bool fgeq(float l, float r) { return (l > r) || feq(l, r); }

}  // namespace careb200
