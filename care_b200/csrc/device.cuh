// device.cuh -- shared types and device helpers of the sm_100a correction path.
//
// Sequences: 2-bit codes A=0,C=1,G=2,T=3 packed 16 per uint32, MSB-first
// (the reference's layout, include/sequencehelpers.hpp:152-187). The aligner
// works on "hi/lo bit planes" held in 32-bit words: plane bit i (MSB-first)
// is the high / low bit of base i (the HiLo layout of
// sequencehelpers.hpp:645-697).
//
// The per-thread helpers are __host__ __device__ so that a host build can
// check them against the CPU oracle; the few intrinsics have host shims.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace careb200 {

#define CB_HD __host__ __device__ __forceinline__

CB_HD uint32_t funnel_l(uint32_t lo, uint32_t hi, int r) {   // high word of (hi:lo) << r
#ifdef __CUDA_ARCH__
    return __funnelshift_l(lo, hi, r);
#else
    return (uint32_t)(((((unsigned long long)hi) << 32) | lo) << (r & 31) >> 32);
#endif
}
CB_HD int popc32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}
CB_HD uint32_t brev32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
#endif
}
CB_HD uint32_t ldg32(const uint32_t* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
// IEEE single operations without contraction (host side is built with
// -ffp-contract=off)
CB_HD float fmul_rn(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
CB_HD float fdiv_rn(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
CB_HD float fsub_rn(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
CB_HD int f2i_rz(float x) {
#ifdef __CUDA_ARCH__
    return __float2int_rz(x);
#else
    return (int)x;
#endif
}

constexpr int kMaxLen = 256;          // longest read the kernels accept
constexpr int kMaxMaps = 48;          // maximum_number_of_maps, include/config.hpp:31

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
    int clf_mode;                     // 0 plain rule, 1 plain + decision rows, 2 network decides
    int clf_min_coverage;             // decision columns below this coverage keep the plain rule
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
    kStatusFeatOverflow = 8,          // decision-column arena too small
};

// MurmurHash3 64-bit finalizer (the published fmix64), as used by the
// reference's minhasher (hpc_helpers hashers.cuh:85-139).
CB_HD unsigned long long murmur64(unsigned long long x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// Reverse complement of a 32-base 2-bit word (reverse the 2-bit groups,
// complement each code).
CB_HD unsigned long long revcomp64(unsigned long long n) {
    n = ((n >> 2) & 0x3333333333333333ull) | ((n & 0x3333333333333333ull) << 2);
    n = ((n >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((n & 0x0F0F0F0F0F0F0F0Full) << 4);
    n = ((n >> 8) & 0x00FF00FF00FF00FFull) | ((n & 0x00FF00FF00FF00FFull) << 8);
    n = ((n >> 16) & 0x0000FFFF0000FFFFull) | ((n & 0x0000FFFF0000FFFFull) << 16);
    n = (n >> 32) | (n << 32);
    return ~n;
}

// k-mer of k bases starting at base pos of a packed sequence (k <= 32).
CB_HD unsigned long long kmer_at(const uint32_t* s, int k, int pos) {
    const int w = pos >> 4, o = pos & 15;
    // up to three 32-bit words cover 32 bases at any offset
    const unsigned long long hi = ((unsigned long long)s[w] << 32) | (unsigned long long)s[w + 1];
    const unsigned long long lo = (unsigned long long)s[w + 2];
    // 96-bit window [hi:64 | lo:32]; take 2k bits starting at bit 2*o from the top
    const unsigned long long top = o ? (hi << (2 * o)) | (lo >> (32 - 2 * o)) : hi;
    return top >> (64 - 2 * k);
}

// 2-bit code of base p of a packed row.
CB_HD uint32_t base_at(const uint32_t* s, int p) {
    return (s[p >> 4] >> (30 - 2 * (p & 15))) & 3u;
}

// Compress the even bits (0,2,...,30) of x into the low 16 bits, order kept.
CB_HD uint32_t even_bits(uint32_t x) {
    x &= 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    x = (x | (x >> 8)) & 0x0000FFFFu;
    return x;
}

// The 2-bit row of a read -> hi/lo bit planes of NW 32-bit words (32 bases
// per word, MSB-first; the reference's HiLo layout, sequencehelpers.hpp:
// 645-697), plus two zero words so that windows may read past the end.
template <int NW>
CB_HD void load_planes(const uint32_t* __restrict__ s, int L,
                                            uint32_t (&hi)[NW + 2], uint32_t (&lo)[NW + 2]) {
    const int nints = (L + 15) >> 4;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const uint32_t x0 = 2 * w < nints ? ldg32(s + 2 * w) : 0u;
        const uint32_t x1 = 2 * w + 1 < nints ? ldg32(s + 2 * w + 1) : 0u;
        uint32_t h = (even_bits(x0 >> 1) << 16) | even_bits(x1 >> 1);
        uint32_t l = (even_bits(x0) << 16) | even_bits(x1);
        const int valid = L - 32 * w;
        const uint32_t m = valid >= 32 ? 0xFFFFFFFFu : (valid <= 0 ? 0u : ~(0xFFFFFFFFu >> valid));
        hi[w] = h & m;
        lo[w] = l & m;
    }
    hi[NW] = hi[NW + 1] = 0u;
    lo[NW] = lo[NW + 1] = 0u;
}

// Planes of the reverse complement of a read of length L: base i of the
// result is the complement of base L-1-i (complement flips both bits).
template <int NW>
CB_HD void revcomp_planes(const uint32_t (&hi)[NW + 2], const uint32_t (&lo)[NW + 2],
                                               int L, uint32_t (&rhi)[NW + 2], uint32_t (&rlo)[NW + 2]) {
#pragma unroll
    for (int j = 0; j < NW; ++j) { rhi[j] = brev32(hi[NW - 1 - j]); rlo[j] = brev32(lo[NW - 1 - j]); }
    rhi[NW] = rhi[NW + 1] = 0u;
    rlo[NW] = rlo[NW + 1] = 0u;
    const int d = 32 * NW - L;            // leading bits that came from padding
    const int dq = d >> 5, dr = d & 31;
#pragma unroll
    for (int step = 0; step < NW; ++step) {
        if (step < dq) {
#pragma unroll
            for (int j = 0; j < NW; ++j) { rhi[j] = rhi[j + 1]; rlo[j] = rlo[j + 1]; }
            rhi[NW] = 0u; rlo[NW] = 0u;
        }
    }
#pragma unroll
    for (int j = 0; j < NW; ++j) {
        rhi[j] = funnel_l(rhi[j + 1], rhi[j], dr);
        rlo[j] = funnel_l(rlo[j + 1], rlo[j], dr);
        const int valid = L - 32 * j;
        const uint32_t m = valid >= 32 ? 0xFFFFFFFFu : (valid <= 0 ? 0u : ~(0xFFFFFFFFu >> valid));
        rhi[j] = (~rhi[j]) & m;
        rlo[j] = (~rlo[j]) & m;
    }
}

struct ShdResult {
    int score, overlap, shift, nops, valid;
};

// Keeps the `valid` leading bits of a 32-bit word (valid in 0..32).
CB_HD uint32_t lead_mask(int valid) {
    return valid >= 32 ? 0xFFFFFFFFu : (valid <= 0 ? 0u : ~(0xFFFFFFFFu >> valid));
}

// Word compares a scan runs (statistics only): WordCount counts them,
// NoCount compiles to nothing.
struct NoCount { CB_HD void add(int) {} };
struct WordCount { int n = 0; CB_HD void add(int k) { n += k; } };

// One scan direction of the shifted Hamming distance. The "shifted" planes S
// slide by t = t0..t1 bases against the "other" planes O, in the reference's
// order and with its pruning (src/cpu_alignment.cpp:247-316):
//   max_errors_excl = min(int(ov * maxErrorRate), best - total + 2*ov);
//   max_errors_excl <= 0 ends the direction; a shift whose mismatch count is
//   below it replaces the best when its score is strictly smaller.
// Mismatches are counted 64 bases at a time (two funnel-shifted 32-bit words
// per plane); further words are only read while the count stays below the
// limit, which decides the same comparisons as the reference's early exit.
// mextab[ov] holds int(float(ov) * maxErrorRate).
template <int NW, class Cnt = NoCount>
CB_HD void shd_scan(uint32_t (&Sh)[NW + 2], uint32_t (&Sl)[NW + 2],
                                         const uint32_t (&Oh)[NW + 2], const uint32_t (&Ol)[NW + 2],
                                         int t0, int t1, int sign, int La, int Lc, int total,
                                         const int* __restrict__ mextab, int& best, int& bestShift,
                                         Cnt* cnt = nullptr) {
    if (t1 < t0) return;
    bool stop = false;
    // overlap at shift t: min(A - t, B) in both directions
    const int A = sign > 0 ? La : Lc, B = sign > 0 ? Lc : La;
    int bt = best - total;
#pragma unroll 1
    for (int w = 0; w <= (t1 >> 5) && !stop; ++w) {
        const int rb = (w == (t0 >> 5)) ? (t0 & 31) : 0;
        const int re = (w == (t1 >> 5)) ? (t1 & 31) : 31;
#pragma unroll 1
        for (int r = rb; r <= re; ++r) {
            const int t = 32 * w + r;
            const int ov = min(A - t, B);
            const int mex = min(mextab[ov], bt + 2 * ov);
            if (mex <= 0) { stop = true; break; }
            uint32_t d0 = (funnel_l(Sh[1], Sh[0], r) ^ Oh[0]) | (funnel_l(Sl[1], Sl[0], r) ^ Ol[0]);
            uint32_t d1 = (funnel_l(Sh[2], Sh[1], r) ^ Oh[1]) | (funnel_l(Sl[2], Sl[1], r) ^ Ol[1]);
            if (ov < 64) { d0 &= lead_mask(ov); d1 &= lead_mask(ov - 32); }
            int mm = popc32(d0) + popc32(d1);
            if (cnt) cnt->add(2);
            if (mm < mex && ov > 64) {
#pragma unroll
                for (int j = 2; j < NW; ++j) {
                    if (32 * j < ov && mm < mex) {
                        uint32_t dj = (funnel_l(Sh[j + 1], Sh[j], r) ^ Oh[j]) |
                                      (funnel_l(Sl[j + 1], Sl[j], r) ^ Ol[j]);
                        dj &= lead_mask(ov - 32 * j);
                        mm += popc32(dj);
                        if (cnt) cnt->add(1);
                    }
                }
            }
            // mm < mex <= best - total + 2*ov: the score improves on the best
            if (mm < mex) {
                bt = mm - 2 * ov;
                best = bt + total;
                bestShift = sign * t;
            }
        }
        // slide the shifted planes by one 32-base word
#pragma unroll
        for (int j = 0; j < NW + 1; ++j) { Sh[j] = Sh[j + 1]; Sl[j] = Sl[j + 1]; }
        Sh[NW + 1] = 0u; Sl[NW + 1] = 0u;
    }
}

// The forward scan of a pair of reads of equal length L, answering both
// directions at once: (A, C) with A as anchor and (C, A) with C as anchor.
// (C, A) at shift -s compares the same bases as (A, C) at s, with the same
// shift range (same length, same minimum overlap), but scans in the order
// 0, -1, ..., -(L-minov), 1, ..., L-minov (in A's shifts). Each direction's
// result is the first shift of its own order among the valid shifts with the
// minimal score, so the scan keeps every shift whose score can tie the best
// (limit best - total + 2*ov + 1, direction ended only when no later shift
// can reach the best) and records the first minimal shift of each order.
// Shift s < 0 has rank -s in the (C, A) order, s > 0 rank (L-minov) + s.
template <int NW, class Cnt = NoCount>
CB_HD void shd_scan_ties(uint32_t (&Sh)[NW + 2], uint32_t (&Sl)[NW + 2],
                         const uint32_t (&Oh)[NW + 2], const uint32_t (&Ol)[NW + 2],
                         int t0, int t1, int sign, int L, int negs, int total,
                         const int* __restrict__ mextab, int& best, int& shiftA, int& shiftB,
                         Cnt* cnt = nullptr) {
    if (t1 < t0) return;
    bool stop = false;
#pragma unroll 1
    for (int w = 0; w <= (t1 >> 5) && !stop; ++w) {
        const int rb = (w == (t0 >> 5)) ? (t0 & 31) : 0;
        const int re = (w == (t1 >> 5)) ? (t1 & 31) : 31;
#pragma unroll 1
        for (int r = rb; r <= re; ++r) {
            const int t = 32 * w + r;
            const int ov = L - t;                       // equal lengths: overlap L - |shift|
            const int mex = min(mextab[ov], best - total + 2 * ov + 1);
            if (mex <= 0) { stop = true; break; }
            uint32_t d0 = (funnel_l(Sh[1], Sh[0], r) ^ Oh[0]) | (funnel_l(Sl[1], Sl[0], r) ^ Ol[0]);
            uint32_t d1 = (funnel_l(Sh[2], Sh[1], r) ^ Oh[1]) | (funnel_l(Sl[2], Sl[1], r) ^ Ol[1]);
            if (ov < 64) { d0 &= lead_mask(ov); d1 &= lead_mask(ov - 32); }
            int mm = popc32(d0) + popc32(d1);
            if (cnt) cnt->add(2);
            if (mm < mex && ov > 64) {
#pragma unroll
                for (int j = 2; j < NW; ++j) {
                    if (32 * j < ov && mm < mex) {
                        uint32_t dj = (funnel_l(Sh[j + 1], Sh[j], r) ^ Oh[j]) |
                                      (funnel_l(Sl[j + 1], Sl[j], r) ^ Ol[j]);
                        dj &= lead_mask(ov - 32 * j);
                        mm += popc32(dj);
                        if (cnt) cnt->add(1);
                    }
                }
            }
            if (mm < mex) {
                const int sc = mm + total - 2 * ov;
                const int s = sign * t;
                if (sc < best) { best = sc; shiftA = s; shiftB = s; }
                else if (sc == best) {
                    const int rs = s <= 0 ? -s : negs + s, rb2 = shiftB <= 0 ? -shiftB : negs + shiftB;
                    if (rs < rb2) shiftB = s;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NW + 1; ++j) { Sh[j] = Sh[j + 1]; Sl[j] = Sl[j + 1]; }
        Sh[NW + 1] = 0u; Sl[NW + 1] = 0u;
    }
}

// Forward alignments of (A, C) and (C, A) for reads of equal length L.
template <int NW, class Cnt = NoCount>
CB_HD void shifted_hamming_pair(const uint32_t (&Ah)[NW + 2], const uint32_t (&Al)[NW + 2],
                                const uint32_t (&Ch)[NW + 2], const uint32_t (&Cl)[NW + 2], int L, int minov,
                                const int* __restrict__ mextab, ShdResult& ac, ShdResult& ca,
                                Cnt* cnt = nullptr) {
    const int total = 2 * L;
    int best = total, shiftA = -L, shiftB = -L;
    uint32_t Sh[NW + 2], Sl[NW + 2];
#pragma unroll 1
    for (int dir = 0; dir < 2; ++dir) {
#pragma unroll
        for (int j = 0; j < NW + 2; ++j) { Sh[j] = dir ? Ch[j] : Ah[j]; Sl[j] = dir ? Cl[j] : Al[j]; }
        if (dir == 0)
            shd_scan_ties<NW>(Sh, Sl, Ch, Cl, 0, L - minov, +1, L, L - minov, total, mextab, best, shiftA, shiftB, cnt);
        else
            shd_scan_ties<NW>(Sh, Sl, Ah, Al, 1, L - minov, -1, L, L - minov, total, mextab, best, shiftA, shiftB, cnt);
    }
    auto fill = [&](ShdResult& res, int shift) {
        res.valid = shift != -L;
        const int cb = max(-shift, 0);
        const int ce = min(L, L - shift);
        res.overlap = ce - cb;
        res.score = best;
        res.shift = shift;
        res.nops = best - total + 2 * res.overlap;
    };
    fill(ac, shiftA);
    fill(ca, shiftB == -L ? -L : -shiftB);
}

// Sum of ceil(v/32) for v = 1..n (0 for n <= 0).
CB_HD int words_prefix(int n) {
    if (n <= 0) return 0;
    const int q = n >> 5, r = n & 31;
    return 16 * q * (q + 1) + (q + 1) * r;
}

// Un-pruned work of one orientation of shifted_hamming: 32-bit word
// compares over every scanned shift, ceil(overlap/32) each. Closed form of
// the two scans above: shifts t = 0..La-minov with overlap min(La-t, Lc),
// then t = 1..Lc-minov with overlap min(La, Lc-t). 743 at La = Lc = 150.
CB_HD int unpruned_words(int La, int Lc, int minov) {
    int w = 0;
    const int T0 = La - minov;
    if (T0 >= 0) {
        const int flat = La >= Lc ? min(T0, La - Lc) + 1 : 0;     // overlap == Lc
        w += flat * ((Lc + 31) >> 5);
        const int top = La - max(0, La - Lc + 1);                 // overlap La - t below that
        if (top >= minov) w += words_prefix(top) - words_prefix(minov - 1);
    }
    const int T1 = Lc - minov;
    if (T1 >= 1) {
        const int flat = Lc > La ? min(T1, Lc - La) : 0;          // overlap == La
        w += flat * ((La + 31) >> 5);
        const int top = Lc - max(1, Lc - La + 1);
        if (top >= minov) w += words_prefix(top) - words_prefix(minov - 1);
    }
    return w;
}

// cpuShiftedHammingDistancePopcount2BitHiLo (src/cpu_alignment.cpp:32-323):
// shifts 0..La-minov (anchor slid against the candidate), then -1..-(Lc-minov)
// (candidate slid against the anchor).
template <int NW, class Cnt = NoCount>
CB_HD ShdResult shifted_hamming(const uint32_t (&Ah)[NW + 2], const uint32_t (&Al)[NW + 2],
                                                     int La, const uint32_t (&Ch)[NW + 2],
                                                     const uint32_t (&Cl)[NW + 2], int Lc, int minov,
                                                     const int* __restrict__ mextab, Cnt* cnt = nullptr) {
    const int total = La + Lc;
    int best = total, bestShift = -Lc;
    uint32_t Sh[NW + 2], Sl[NW + 2];
#pragma unroll 1
    for (int dir = 0; dir < 2; ++dir) {
#pragma unroll
        for (int j = 0; j < NW + 2; ++j) { Sh[j] = dir ? Ch[j] : Ah[j]; Sl[j] = dir ? Cl[j] : Al[j]; }
        if (dir == 0) shd_scan<NW>(Sh, Sl, Ch, Cl, 0, La - minov, +1, La, Lc, total, mextab, best, bestShift, cnt);
        else shd_scan<NW>(Sh, Sl, Ah, Al, 1, Lc - minov, -1, La, Lc, total, mextab, best, bestShift, cnt);
    }
    ShdResult res;
    res.valid = bestShift != -Lc;
    const int cb = max(-bestShift, 0);
    const int ce = min(Lc, La - bestShift);
    res.overlap = ce - cb;
    res.score = best;
    res.shift = bestShift;
    res.nops = best - total + 2 * res.overlap;
    return res;
}

// chooseBestAlignmentOrientation (include/alignmentorientation.hpp:12-92).
CB_HD int choose_orientation(const ShdResult& f, const ShdResult& r, int La,
                                                  float min_overlap_ratio, int min_overlap,
                                                  float maxErrorRate) {
    int ret = 3;
    const int lo = f2i_rz(fmul_rn((float)La, min_overlap_ratio));
    const int mo = lo > min_overlap ? lo : min_overlap;
    if (f.valid && f.overlap >= mo) {
        if (r.valid && r.overlap >= mo) {
            const float ratio = fdiv_rn((float)f.nops, (float)f.overlap);
            const float rratio = fdiv_rn((float)r.nops, (float)r.overlap);
            if (ratio < rratio) { if (ratio < maxErrorRate) ret = 1; }
            else if (rratio < ratio) { if (rratio < maxErrorRate) ret = 2; }
            else if (ratio < maxErrorRate) ret = f.overlap > r.overlap ? 1 : 2;
        } else if (fdiv_rn((float)f.nops, (float)f.overlap) < maxErrorRate) ret = 1;
    } else if (r.valid && r.overlap >= mo) {
        if (fdiv_rn((float)r.nops, (float)r.overlap) < maxErrorRate) ret = 2;
    }
    return ret;
}

// feq / fleq / fgeq (include/hostdevicefunctions.cuh:9-29).
CB_HD bool feq(float l, float r) {
    const float d = fsub_rn(l, r);
    return (d < 0 ? -d : d) < 1e-5f;
}
CB_HD bool fleq(float l, float r) { return (l < r) || feq(l, r); }
CB_HD bool fgeq(float l, float r) { return (l > r) || feq(l, r); }

}  // namespace careb200
