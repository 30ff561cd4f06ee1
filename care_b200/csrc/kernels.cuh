// kernels.cuh -- the three device stages of one correction batch.
//
//   k_candidates : minhash signature + table lookup + de-duplication
//                  (one CTA per anchor)
//   k_align      : shifted Hamming distance, both strands, orientation,
//                  pair flag (one thread per (anchor, candidate) pair)
//   k_msa        : alignment filters, MSA build/refine, consensus
//                  correction of anchor and candidates (one CTA per anchor)
#pragma once
#include <type_traits>
#include "device.cuh"

namespace careb200 {

__constant__ float c_qweight[256];    // QualityScoreConversion table (qualityscoreweights.hpp:16-31)

// ---------------------------------------------------------------------------
// Stage 1: candidate read ids per anchor.
//   CPUSequenceHasher::hashInto       include/cpusequencehasher.hpp:88-125
//   forEachEncodedCanonicalKmer...    include/sequencehelpers.hpp:844-926
//   OrdinaryCpuMinhasher::determineNumValues/retrieveValues/queryMap
//                                     include/ordinaryminhasher.hpp:135-221,437-449
//   determineCandidateReadIds         include/corrector.hpp:571-650
// The table-major concatenation is followed by sort+unique in the reference;
// here a shared-memory hash set removes duplicates and a bitonic sort orders
// the (few) unique ids: same set, same ascending order.
// ---------------------------------------------------------------------------
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

struct CandSmem {
    // dynamic shared memory layout, all offsets in bytes
    static __host__ __device__ size_t canon(int) { return 0; }
    static __host__ __device__ size_t partial(int maxlen) { return (size_t)(maxlen + 8) * 8; }
    static __host__ __device__ size_t seq(int maxlen, int groups, int maps) {
        return partial(maxlen) + (size_t)groups * maps * 8;
    }
    static __host__ __device__ size_t qinfo(int maxlen, int groups, int maps, int pitch) {
        return seq(maxlen, groups, maps) + (size_t)(pitch + 4) * 4;
    }
    static __host__ __device__ size_t set(int maxlen, int groups, int maps, int pitch) {
        return qinfo(maxlen, groups, maps, pitch) + (size_t)(3 * kMaxMaps + 8) * 4;
    }
    static __host__ __device__ size_t total(int maxlen, int groups, int maps, int pitch, int setcap) {
        return set(maxlen, groups, maps, pitch) + (size_t)setcap * 4 * 2;
    }
};

// The candidate list of anchor ai, by one CTA. The de-duplication set has
// 2^sl2 entries, sl2 the smallest with 2^sl2 >= 2T (T ids retrieved), at most
// 2^set_log2. With a spill list the capacity is small (most anchors hold a few
// dozen unique ids among hundreds retrieved) and an anchor with more than
// half as many unique ids is appended to the list instead: its segment is
// then written by k_candidates_spill with a set large enough for every id.
template <int BLOCK>
__device__ __forceinline__ void candidates_of(
    const DevOptions& o, const DevReads& r, const TableDesc* __restrict__ td, const Slot* __restrict__ slots,
    const uint32_t* __restrict__ values, const unsigned long long* __restrict__ sig, uint32_t first, uint32_t ai,
    int set_log2, uint32_t* __restrict__ spill_list, unsigned int* __restrict__ spill_n,
    uint32_t* __restrict__ cand_ids, uint32_t* __restrict__ cand_anchor, uint32_t* __restrict__ seg_off,
    uint32_t* __restrict__ seg_cnt, unsigned long long* __restrict__ arena_count, unsigned long long arena_cap,
    int* __restrict__ status, unsigned char* smem, uint32_t& s_unique, uint32_t& s_ins, uint32_t& s_full,
    unsigned long long& s_base) {
    const int tid = threadIdx.x;
    const uint32_t a = first + ai;
    const int h = o.num_maps;
    const int groups = BLOCK / h;
    const int setcap = 1 << set_log2;
    unsigned long long* canon = (unsigned long long*)(smem + CandSmem::canon(r.max_len));
    unsigned long long* partial = (unsigned long long*)(smem + CandSmem::partial(r.max_len));
    uint32_t* sseq = (uint32_t*)(smem + CandSmem::seq(r.max_len, groups, h));
    uint32_t* qoff = (uint32_t*)(smem + CandSmem::qinfo(r.max_len, groups, h, r.seq_pitch));
    uint32_t* qcnt = qoff + kMaxMaps;
    uint32_t* qpre = qcnt + kMaxMaps;              // kMaxMaps + 1 entries
    uint32_t* set = (uint32_t*)(smem + CandSmem::set(r.max_len, groups, h, r.seq_pitch));
    uint32_t* list = set + setcap;

    const int L = r.len[a];
    const bool skip = (o.exclude_ambiguous && r.ambig[a]) || L < o.k;
    if (skip) {
        if (tid == 0) { seg_off[ai] = 0; seg_cnt[ai] = 0; }
        return;
    }
    // the anchor's signature: resident (computed once per read storage by
    // k_signatures), or hashed here
    if (!sig) {
        // anchor row into shared memory, two zero words of padding for kmer_at
        const uint32_t* arow = r.seq + (size_t)a * r.seq_pitch;
        for (int i = tid; i < r.seq_pitch + 2; i += BLOCK) sseq[i] = i < r.seq_pitch ? __ldg(arow + i) : 0u;
        __syncthreads();

        // canonical k-mers
        const int npos = L - o.k + 1;
        const int rcshift = 64 - 2 * o.k;
        for (int p = tid; p < npos; p += BLOCK) {
            const unsigned long long fw = kmer_at(sseq, o.k, p);
            const unsigned long long rv = revcomp64(fw) >> rcshift;
            canon[p] = fw < rv ? fw : rv;
        }
        __syncthreads();

        // per map: min over k-mers of murmur64(kmer + map)
        {
            const int m = tid % h, g = tid / h;
            if (g < groups) {
                unsigned long long mn = ~0ull;
                for (int p = g; p < npos; p += groups) {
                    const unsigned long long v = murmur64(canon[p] + (unsigned long long)m);
                    mn = v < mn ? v : mn;
                }
                partial[g * h + m] = mn;
            }
        }
        __syncthreads();
    }

    // table lookup (linear probing from murmur64(key))
    if (tid < h) {
        unsigned long long key = ~0ull;
        if (sig) {
            key = __ldg(sig + (size_t)a * h + tid);
        } else {
            for (int g = 0; g < groups; ++g) { const unsigned long long v = partial[g * h + tid]; key = v < key ? v : key; }
            key &= o.kmer_mask;
        }
        const TableDesc d = td[tid];
        uint32_t pos = (uint32_t)murmur64(key) & d.mask;
        uint32_t off = 0, cnt = 0;
        for (uint32_t probe = 0; probe <= d.mask; ++probe) {
            const Slot sl = slots[d.slot_base + pos];
            if (sl.count == 0) break;
            if (sl.key == key) { off = sl.offset; cnt = sl.count; break; }
            pos = (pos + 1) & d.mask;
        }
        if ((int)cnt > o.threshold) cnt = 0;      // queryMap :443-446
        qoff[tid] = (uint32_t)d.value_base + off;
        qcnt[tid] = cnt;
    }
    if (tid == 0) { s_unique = 0; s_ins = 0; s_full = 0; }
    __syncthreads();
    if (tid < 32) {                                  // offsets of the maps' runs: warp scan, two maps per lane
        const uint32_t c0 = tid < h ? qcnt[tid] : 0u, c1 = tid + 32 < h ? qcnt[tid + 32] : 0u;
        uint32_t s0 = c0, s1 = c1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t0 = __shfl_up_sync(0xffffffffu, s0, d), t1 = __shfl_up_sync(0xffffffffu, s1, d);
            if (tid >= d) { s0 += t0; s1 += t1; }
        }
        const uint32_t tot0 = __shfl_sync(0xffffffffu, s0, 31);
        if (tid < h) qpre[tid] = s0 - c0;
        if (tid + 32 < h) qpre[tid + 32] = tot0 + s1 - c1;
        if (tid == 31) qpre[h] = tot0 + s1;
    }
    __syncthreads();

    // the hash set is sized for the ids actually retrieved: a power of two
    // >= 2 * T (at least 64), within the allocated capacity
    const uint32_t T = qpre[h];
    int sl2 = 6;
    while (sl2 < set_log2 && (1u << sl2) < 2 * T) ++sl2;
    const int scap = 1 << sl2;
    // without a spill list the set always has room (2^set_log2 > h * threshold >= T)
    const uint32_t limit = spill_list ? (uint32_t)scap / 2 : 0xffffffffu;
    for (int i = tid; i < scap; i += BLOCK) set[i] = kEmpty;
    __syncthreads();

    // insert all retrieved ids into the shared hash set, eight loads in
    // flight per thread ahead of their inserts
    constexpr int kInFlight = 8;
    for (uint32_t e0 = 0; e0 < T; e0 += BLOCK * kInFlight) {
        uint32_t ids[kInFlight];
#pragma unroll
        for (int k = 0; k < kInFlight; ++k) {
            const uint32_t e = e0 + (uint32_t)(k * BLOCK + tid);
            ids[k] = kEmpty;
            if (e < T) {
                int lo = 0, hi = h - 1;             // map of element e
                while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (qpre[mid] <= e) lo = mid; else hi = mid - 1; }
                ids[k] = __ldg(values + qoff[lo] + (e - qpre[lo]));
            }
        }
#pragma unroll
        for (int k = 0; k < kInFlight; ++k) {
            const uint32_t id = ids[k];                // read ids are < 2^32 - 1: kEmpty marks none
            if (id == kEmpty || *(volatile uint32_t*)&s_full) continue;
            uint32_t pos = (id * 2654435761u) >> (32 - sl2);
            bool placed = false;
            for (int probe = 0; probe < scap; ++probe) {
                const uint32_t prev = atomicCAS(&set[pos], kEmpty, id);
                if (prev == kEmpty) {
                    placed = true;
                    if (atomicAdd(&s_ins, 1u) >= limit) s_full = 1;
                    break;
                }
                if (prev == id) { placed = true; break; }
                pos = (pos + 1) & (scap - 1);
            }
            if (!placed) s_full = 1;
        }
    }
    __syncthreads();
    if (s_full) {                                   // block-uniform: the second pass takes the anchor
        if (tid == 0) spill_list[atomicAdd(spill_n, 1u)] = ai;
        return;
    }

    // unique ids minus the anchor itself and (optionally) ambiguous reads
    for (int i = tid; i < scap; i += BLOCK) {
        const uint32_t v = set[i];
        if (v != kEmpty && v != a && !(o.exclude_ambiguous && r.ambig[v])) list[atomicAdd(&s_unique, 1u)] = v;
    }
    __syncthreads();
    const uint32_t U = s_unique;
    uint32_t P = 32;
    while (P < U) P <<= 1;
    for (uint32_t i = U + tid; i < P; i += BLOCK) list[i] = kEmpty;
    __syncthreads();
    // bitonic sort of list[0..P): exchanges across warps (partner distance
    // >= 32) through shared memory, one barrier each; the exchanges within a
    // warp (distance < 32) of a merge level in registers with shuffles
    const int wid = tid >> 5, ln = tid & 31;
    for (uint32_t kk = 2; kk <= P; kk <<= 1) {
        for (uint32_t j = kk >> 1; j >= 32; j >>= 1) {
            for (uint32_t i = tid; i < P; i += BLOCK) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const uint32_t x = list[i], y = list[ixj];
                    const bool up = (i & kk) == 0;
                    if ((x > y) == up) { list[i] = y; list[ixj] = x; }
                }
            }
            __syncthreads();
        }
        for (uint32_t i0 = 32u * wid; i0 < P; i0 += BLOCK) {      // warp-uniform
            const uint32_t i = i0 + ln;
            uint32_t x = list[i];
            const bool up = (i & kk) == 0;
            for (uint32_t j = min(kk >> 1, 16u); j > 0; j >>= 1) {
                const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
                x = (up == ((i & j) == 0)) ? min(x, y) : max(x, y);
            }
            list[i] = x;
        }
        __syncthreads();
    }
    if (tid == 0) s_base = atomicAdd(arena_count, (unsigned long long)U);
    __syncthreads();
    const unsigned long long base = s_base;
    if (tid == 0) { seg_off[ai] = (uint32_t)base; seg_cnt[ai] = U; }
    if (base + U > arena_cap) {
        if (tid == 0) atomicOr(status, kStatusCandOverflow);
        return;
    }
    for (uint32_t i = tid; i < U; i += BLOCK) { cand_ids[base + i] = list[i]; cand_anchor[base + i] = ai; }
}

// One anchor per CTA, the set capacity 2^set_log2 (small when spill_list is
// given: the anchors that overflow it are listed for k_candidates_spill).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_candidates(DevOptions o, DevReads r, const TableDesc* __restrict__ td, const Slot* __restrict__ slots,
             const uint32_t* __restrict__ values, const unsigned long long* __restrict__ sig,
             uint32_t first, uint32_t count, int set_log2, uint32_t* __restrict__ spill_list,
             unsigned int* __restrict__ spill_n, uint32_t* __restrict__ cand_ids, uint32_t* __restrict__ cand_anchor,
             uint32_t* __restrict__ seg_off, uint32_t* __restrict__ seg_cnt,
             unsigned long long* __restrict__ arena_count, unsigned long long arena_cap,
             int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_unique, s_ins, s_full;
    __shared__ unsigned long long s_base;
    if (blockIdx.x >= count) return;
    candidates_of<BLOCK>(o, r, td, slots, values, sig, first, blockIdx.x, set_log2, spill_list, spill_n, cand_ids,
                         cand_anchor, seg_off, seg_cnt, arena_count, arena_cap, status, smem, s_unique, s_ins,
                         s_full, s_base);
}

// The listed anchors with a set for every retrieved id (persistent CTAs).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_candidates_spill(DevOptions o, DevReads r, const TableDesc* __restrict__ td, const Slot* __restrict__ slots,
                   const uint32_t* __restrict__ values, const unsigned long long* __restrict__ sig, uint32_t first,
                   int set_log2, const uint32_t* __restrict__ spill_list, const unsigned int* __restrict__ spill_n,
                   uint32_t* __restrict__ cand_ids, uint32_t* __restrict__ cand_anchor,
                   uint32_t* __restrict__ seg_off, uint32_t* __restrict__ seg_cnt,
                   unsigned long long* __restrict__ arena_count, unsigned long long arena_cap,
                   int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_unique, s_ins, s_full;
    __shared__ unsigned long long s_base;
    const unsigned int n = *spill_n;
    for (unsigned int k = blockIdx.x; k < n; k += gridDim.x) {
        candidates_of<BLOCK>(o, r, td, slots, values, sig, first, spill_list[k], set_log2, nullptr, nullptr,
                             cand_ids, cand_anchor, seg_off, seg_cnt, arena_count, arena_cap, status, smem,
                             s_unique, s_ins, s_full, s_base);
        __syncthreads();                            // the next anchor reuses the shared state
    }
}

// ---------------------------------------------------------------------------
// Stage 2: alignment of every (anchor, candidate) pair, both strands.
//   getCandidateAlignments            include/corrector.hpp:925-979
//   cpuShiftedHammingDistance...      src/cpu_alignment.cpp:32-323
//   chooseBestAlignmentOrientation    include/alignmentorientation.hpp:72-92
//   computePairFlags                  include/corrector.hpp:763-807 (PE)
// ---------------------------------------------------------------------------
constexpr uint32_t kNoMirror = 0xffffffffu;

// Mirror pairs. When candidate c of anchor a is itself an anchor of the
// batch, has a's length and holds a among its candidates, the pairs (a, c)
// and (c, a) share their scans: the reverse-complement alignments are the
// same (same shift, overlap and mismatches) and both forward alignments come
// from one tie-aware scan (shifted_hamming_pair). The pair with a < c leads
// and computes both results; its mirror is skipped. Work list: leaders
// {pair, mirror} from the front, single pairs {pair, kNoMirror} from the
// back (index total-1 down), counts in work_n[0] and work_n[1].
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_pair_mirror(DevReads r, uint32_t first, uint32_t count, const uint32_t* __restrict__ cand_ids,
              const uint32_t* __restrict__ cand_anchor, const uint32_t* __restrict__ seg_off,
              const uint32_t* __restrict__ seg_cnt, const unsigned long long* __restrict__ total_ptr,
              unsigned long long arena_cap, const int* __restrict__ status, const uint32_t* __restrict__ pair_order,
              uint2* __restrict__ work, unsigned int* __restrict__ work_n) {
    if (*status & kStatusCandOverflow) return;
    const unsigned long long total = *total_ptr;
    if (total > arena_cap) return;
    const unsigned long long slot = (unsigned long long)blockIdx.x * BLOCK + threadIdx.x;
    if (slot - (threadIdx.x & 31) >= total) return;          // whole warp past the end
    int kind = 0;                                            // 1 leader, 2 single
    uint32_t i = 0, j = kNoMirror;
    if (slot < total) {
        i = pair_order ? pair_order[slot] : (uint32_t)slot;
        const uint32_t a = first + cand_anchor[i];
        const uint32_t c = cand_ids[i];
        kind = 2;
        if (c - first < count && r.len[a] == r.len[c]) {
            const uint32_t ci = c - first, off = seg_off[ci], cnt = seg_cnt[ci];
            uint32_t lo = 0, hi = cnt;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (cand_ids[off + mid] < a) lo = mid + 1; else hi = mid;
            }
            if (lo < cnt && cand_ids[off + lo] == a) {
                j = off + lo;
                kind = a < c ? 1 : 0;
            }
        }
    }
    const unsigned ln = threadIdx.x & 31, below = (1u << ln) - 1u;
    const unsigned ml = __ballot_sync(0xffffffffu, kind == 1), ms = __ballot_sync(0xffffffffu, kind == 2);
    unsigned bl = 0, bs = 0;
    if (ln == 0) {
        if (ml) bl = atomicAdd(&work_n[0], (unsigned)__popc(ml));
        if (ms) bs = atomicAdd(&work_n[1], (unsigned)__popc(ms));
    }
    bl = __shfl_sync(0xffffffffu, bl, 0);
    bs = __shfl_sync(0xffffffffu, bs, 0);
    if (kind == 1) work[bl + __popc(ml & below)] = make_uint2(i, j);
    if (kind == 2) work[total - 1 - (bs + __popc(ms & below))] = make_uint2(i, kNoMirror);
}

// Candidate c's pair flag: c's mate is a candidate of the anchor's mate
// (equivalent to flagPairedCandidates, include/util.hpp:1016-1197).
__device__ __forceinline__ uint8_t mate_flag(const uint32_t* __restrict__ cand_ids, const uint32_t* __restrict__ seg_off,
                       const uint32_t* __restrict__ seg_cnt, uint32_t ai, uint32_t c) {
    const uint32_t mi = ai ^ 1u;
    const uint32_t moff = seg_off[mi], mcnt = seg_cnt[mi];
    const uint32_t target = c ^ 1u;
    uint32_t lo2 = 0, hi2 = mcnt;
    while (lo2 < hi2) {
        const uint32_t mid = (lo2 + hi2) >> 1;
        if (cand_ids[moff + mid] < target) lo2 = mid + 1; else hi2 = mid;
    }
    return (lo2 < mcnt && cand_ids[moff + lo2] == target) ? 1 : 0;
}

// CNT: the statistics form, which also adds the 32-bit word compares its
// scans actually run (after the early exits) to run_count.
// One alignment work item (slot of the mirror work list, of pair_order from
// `base`, or the pair itself): both orientations, the orientation choice and
// the AlignRes (a mirrored pair writes both). false past the work list.
template <int NW, bool CNT>
__device__ __forceinline__ bool
align_item(const DevOptions& o, const DevReads& r, uint32_t first, const uint32_t* __restrict__ cand_ids,
           const uint32_t* __restrict__ cand_anchor, const uint32_t* __restrict__ seg_off,
           const uint32_t* __restrict__ seg_cnt, unsigned long long total, AlignRes* __restrict__ out,
           unsigned long long* __restrict__ work_count, const uint32_t* __restrict__ pair_order,
           unsigned long long base, const uint2* __restrict__ work, const unsigned int* __restrict__ work_n,
           unsigned long long* __restrict__ run_count, const int* s_mex, unsigned long long slot) {
    using Cnt = typename std::conditional<CNT, WordCount, NoCount>::type;
    Cnt wc;
    unsigned long long i;
    uint32_t j = kNoMirror;
    if (work) {                        // mirror work list (k_pair_mirror)
        const unsigned nl = work_n[0], ns = work_n[1];
        if (slot >= (unsigned long long)nl + ns) return false;
        const uint2 w = slot < nl ? work[slot] : work[total - 1 - (slot - nl)];
        i = w.x;
        j = w.y;
    } else {
        i = pair_order ? pair_order[base + slot] : slot;
    }
    const uint32_t ai = cand_anchor[i];
    const uint32_t a = first + ai;
    const uint32_t c = cand_ids[i];
    const int La = r.len[a], Lc = r.len[c];
    uint32_t Ah[NW + 2], Al[NW + 2], Ch[NW + 2], Cl[NW + 2];
    load_planes<NW>(r.seq + (size_t)a * r.seq_pitch, La, Ah, Al);
    load_planes<NW>(r.seq + (size_t)c * r.seq_pitch, Lc, Ch, Cl);
    const int lo = __float2int_rz(__fmul_rn((float)La, o.min_overlap_ratio));
    const int minov = o.min_overlap > lo ? o.min_overlap : lo;
    if (work_count) {                 // un-pruned word compares of the scans run here (roofline work)
        const unsigned m = __activemask();
        const unsigned ws = __reduce_add_sync(m, (unsigned)(2 * unpruned_words(La, Lc, minov)));
        if ((int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(work_count, (unsigned long long)ws);
    }
    ShdResult f, g;                   // g: forward alignment of the mirror pair (c, a)
    if (j != kNoMirror) shifted_hamming_pair<NW, Cnt>(Ah, Al, Ch, Cl, La, minov, s_mex, f, g, &wc);
    else f = shifted_hamming<NW, Cnt>(Ah, Al, La, Ch, Cl, Lc, minov, s_mex, &wc);
    uint32_t Rh[NW + 2], Rl[NW + 2];
    revcomp_planes<NW>(Ch, Cl, Lc, Rh, Rl);
    const ShdResult rc = shifted_hamming<NW, Cnt>(Ah, Al, La, Rh, Rl, Lc, minov, s_mex, &wc);
    if constexpr (CNT) {
        const unsigned m = __activemask();
        const unsigned ws = __reduce_add_sync(m, (unsigned)wc.n);
        if ((int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(run_count, (unsigned long long)ws);
    }
    const float ler = __fmul_rn(o.estimated_errorrate, 4.0f);
    auto result = [&](const ShdResult& fw, uint32_t anchor_index, uint32_t cand) {
        const int orient = choose_orientation(fw, rc, La, o.min_overlap_ratio, o.min_overlap, ler);
        AlignRes res;
        const ShdResult& b = orient == 2 ? rc : fw;
        res.shift = (int16_t)b.shift;
        res.overlap = (int16_t)b.overlap;
        res.nops = (int16_t)b.nops;
        res.orient = (uint8_t)orient;
        res.paired = o.paired_end ? mate_flag(cand_ids, seg_off, seg_cnt, anchor_index, cand) : 0;
        return res;
    };
    out[i] = result(f, ai, c);
    if (j != kNoMirror) out[j] = result(g, c - first, a);
    return true;
}

template <int BLOCK>
__device__ __forceinline__ void align_mex_table(const DevOptions& o, int* s_mex) {
    // int(float(ov) * maxErrorRate), the first term of max_errors_excl
    for (int i = threadIdx.x; i <= kMaxLen; i += BLOCK) s_mex[i] = __float2int_rz(__fmul_rn((float)i, o.max_error_rate));
    __syncthreads();
}

template <int BLOCK, int NW, bool CNT = false>
__global__ void __launch_bounds__(BLOCK)
k_align(DevOptions o, DevReads r, uint32_t first, const uint32_t* __restrict__ cand_ids,
        const uint32_t* __restrict__ cand_anchor, const uint32_t* __restrict__ seg_off,
        const uint32_t* __restrict__ seg_cnt, const unsigned long long* __restrict__ total_ptr,
        unsigned long long arena_cap, const int* __restrict__ status, AlignRes* __restrict__ out,
        unsigned long long* __restrict__ work_count, const uint32_t* __restrict__ pair_order,
        const uint2* __restrict__ work, const unsigned int* __restrict__ work_n,
        unsigned long long* __restrict__ run_count) {
    __shared__ int s_mex[kMaxLen + 1];
    align_mex_table<BLOCK>(o, s_mex);
    // an overflowed candidate arena holds unwritten entries: the batch is
    // repeated with a larger arena, nothing here may read them
    if (*status & kStatusCandOverflow) return;
    const unsigned long long slot = (unsigned long long)blockIdx.x * BLOCK + threadIdx.x;
    const unsigned long long total = *total_ptr;
    if (total > arena_cap || slot >= total) return;
    align_item<NW, CNT>(o, r, first, cand_ids, cand_anchor, seg_off, seg_cnt, total, out, work_count, pair_order, 0,
                        work, work_n, run_count, s_mex, slot);
}

// One length class of the batch's pairs (cls = {offset in the class list,
// pairs}, k_pair_class_*): resident blocks stride over its pairs, with the
// register budget of the class's plane width.
template <int BLOCK, int NW, bool CNT = false>
__global__ void __launch_bounds__(BLOCK, (NW <= 5 ? 1024 : 768) / BLOCK)
k_align_class(DevOptions o, DevReads r, uint32_t first, const uint32_t* __restrict__ cand_ids,
              const uint32_t* __restrict__ cand_anchor, const uint32_t* __restrict__ seg_off,
              const uint32_t* __restrict__ seg_cnt, const unsigned long long* __restrict__ total_ptr,
              unsigned long long arena_cap, const int* __restrict__ status, AlignRes* __restrict__ out,
              unsigned long long* __restrict__ work_count, const uint32_t* __restrict__ class_list,
              const uint2* __restrict__ cls, unsigned long long* __restrict__ run_count) {
    __shared__ int s_mex[kMaxLen + 1];
    align_mex_table<BLOCK>(o, s_mex);
    if (*status & kStatusCandOverflow) return;
    const unsigned long long total = *total_ptr;
    if (total > arena_cap) return;
    const unsigned long long n = cls->y, base = cls->x;
#pragma unroll 1
    for (unsigned long long slot = (unsigned long long)blockIdx.x * BLOCK + threadIdx.x; slot < n;
         slot += (unsigned long long)gridDim.x * BLOCK)
        align_item<NW, CNT>(o, r, first, cand_ids, cand_anchor, seg_off, seg_cnt, total, out, work_count, class_list,
                            base, nullptr, nullptr, run_count, s_mex, slot);
}

// ---------------------------------------------------------------------------
// Warp-cooperative alignment: one warp per work item, lane r of the warp
// takes shift 32*w + r of each group w of 32 shifts (the funnel shift amount
// is the lane; the planes slide by one word per group, as in shd_scan).
// Every lane counts its shift's mismatches up to its own limit
// min(int(ov * maxErrorRate), best - total + 2*ov), with `best` the score
// found by the earlier groups, and the warp keeps the smallest key
// (score << 10 | rank of the shift in the scan order). The result is the
// first shift in scan order with the smallest score among the shifts whose
// mismatches are below int(ov * maxErrorRate): the same shift the sequential
// scan with early exits returns (src/cpu_alignment.cpp:247-316). A direction
// ends at the first group whose leading shift can no longer reach the best
// (its limit is <= 0 and the limit does not grow along a direction).
// TIES: the equal-length pair form (both directions of a mirrored pair, as
// shd_scan_ties): ties with the best are kept (limit + 1) and a second key
// ranks the shifts in the order of the (C, A) scan.
constexpr unsigned kKeyRankBits = 10;          // ranks and scores stay below 1024 (reads <= 256 bases)
constexpr unsigned kKeyRankMask = (1u << kKeyRankBits) - 1u;

// D0: shifts of the first direction (its ranks are t, the second's D0 + t - 1);
// negs: the (C, A) order's count of shifts <= 0 after 0 (TIES).
template <int NW, bool TIES, class Cnt>
__device__ __forceinline__ void shd_scan_lanes(uint32_t (&Sh)[NW + 2], uint32_t (&Sl)[NW + 2],
                                               const uint32_t (&Oh)[NW + 2], const uint32_t (&Ol)[NW + 2],
                                               int t0, int t1, int dir, int La, int Lc, int total, int D0,
                                               int negs, const int* __restrict__ mextab, unsigned& keyA,
                                               unsigned& keyB, Cnt* cnt) {
    if (t1 < t0) return;
    const int lane = threadIdx.x & 31;
    const int tie = TIES ? 1 : 0;
    auto overlap = [&](int t) { return dir == 0 ? min(La - t, Lc) : min(La, Lc - t); };
#pragma unroll 1
    for (int w = 0; w <= (t1 >> 5); ++w) {
        const int t = 32 * w + lane;
        const int best = (int)(keyA >> kKeyRankBits);
        unsigned ka = 0xFFFFFFFFu, kb = 0xFFFFFFFFu;
        if (t >= t0 && t <= t1) {
            const int ov = overlap(t);
            const int mex = min(mextab[ov], best - total + 2 * ov + tie);
            if (mex > 0) {
                const int r = lane;
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
                    const unsigned sc = (unsigned)(mm + total - 2 * ov) << kKeyRankBits;
                    ka = sc | (unsigned)(dir == 0 ? t : D0 + t - 1);
                    if constexpr (TIES) kb = sc | (unsigned)(dir == 0 ? (t == 0 ? 0 : negs + t) : t);
                }
            }
        }
        keyA = min(keyA, __reduce_min_sync(0xffffffffu, ka));
        if constexpr (TIES) keyB = min(keyB, __reduce_min_sync(0xffffffffu, kb));
        const int tn = 32 * (w + 1);
        if (tn > t1) break;
        {   // end of the direction: the next group's first shift cannot reach the best
            const int ovn = overlap(tn);
            if (min(mextab[ovn], (int)(keyA >> kKeyRankBits) - total + 2 * ovn + tie) <= 0) break;
        }
#pragma unroll
        for (int j = 0; j < NW + 1; ++j) { Sh[j] = Sh[j + 1]; Sl[j] = Sl[j + 1]; }
        Sh[NW + 1] = 0u; Sl[NW + 1] = 0u;
    }
}

// ShdResult of a scan from its best key: shift of rank `rank`, the overlap,
// score and mismatches (nOps) of that shift.
__device__ __forceinline__ ShdResult shd_from_shift(int shift, int score, int La, int Lc) {
    ShdResult res;
    res.valid = shift != -Lc;
    const int cb = max(-shift, 0);
    const int ce = min(Lc, La - shift);
    res.overlap = ce - cb;
    res.score = score;
    res.shift = shift;
    res.nops = score - (La + Lc) + 2 * res.overlap;
    return res;
}

// shifted_hamming with the warp: every lane returns the same result.
template <int NW, class Cnt>
__device__ __forceinline__ ShdResult shifted_hamming_lanes(const uint32_t (&Ah)[NW + 2], const uint32_t (&Al)[NW + 2],
                                                           int La, const uint32_t (&Ch)[NW + 2],
                                                           const uint32_t (&Cl)[NW + 2], int Lc, int minov,
                                                           const int* __restrict__ mextab, Cnt* cnt) {
    const int total = La + Lc;
    const int T0 = La - minov;
    const int D0 = T0 + 1 > 0 ? T0 + 1 : 0;      // shifts of the first direction: ranks 0..D0-1
    unsigned keyA = ((unsigned)total << kKeyRankBits) | kKeyRankMask, keyB = 0xFFFFFFFFu;
    uint32_t Sh[NW + 2], Sl[NW + 2];
#pragma unroll 1
    for (int dir = 0; dir < 2; ++dir) {
#pragma unroll
        for (int j = 0; j < NW + 2; ++j) { Sh[j] = dir ? Ch[j] : Ah[j]; Sl[j] = dir ? Cl[j] : Al[j]; }
        if (dir == 0) shd_scan_lanes<NW, false>(Sh, Sl, Ch, Cl, 0, T0, 0, La, Lc, total, D0, 0, mextab, keyA, keyB, cnt);
        else shd_scan_lanes<NW, false>(Sh, Sl, Ah, Al, 1, Lc - minov, 1, La, Lc, total, D0, 0, mextab, keyA, keyB, cnt);
    }
    const int score = (int)(keyA >> kKeyRankBits), rank = (int)(keyA & kKeyRankMask);
    const int shift = score >= total ? -Lc : (rank < D0 ? rank : -(rank - D0 + 1));
    return shd_from_shift(shift, score, La, Lc);
}

// shifted_hamming_pair with the warp: forward (A, C) and (C, A) of a pair of
// equal length L.
template <int NW, class Cnt>
__device__ __forceinline__ void shifted_hamming_pair_lanes(const uint32_t (&Ah)[NW + 2], const uint32_t (&Al)[NW + 2],
                                                           const uint32_t (&Ch)[NW + 2], const uint32_t (&Cl)[NW + 2],
                                                           int L, int minov, const int* __restrict__ mextab,
                                                           ShdResult& ac, ShdResult& ca, Cnt* cnt) {
    const int total = 2 * L;
    const int T = L - minov;
    unsigned keyA = ((unsigned)total << kKeyRankBits) | kKeyRankMask, keyB = keyA;
    uint32_t Sh[NW + 2], Sl[NW + 2];
#pragma unroll 1
    for (int dir = 0; dir < 2; ++dir) {
#pragma unroll
        for (int j = 0; j < NW + 2; ++j) { Sh[j] = dir ? Ch[j] : Ah[j]; Sl[j] = dir ? Cl[j] : Al[j]; }
        if (dir == 0) shd_scan_lanes<NW, true>(Sh, Sl, Ch, Cl, 0, T, 0, L, L, total, T + 1, T, mextab, keyA, keyB, cnt);
        else shd_scan_lanes<NW, true>(Sh, Sl, Ah, Al, 1, T, 1, L, L, total, T + 1, T, mextab, keyA, keyB, cnt);
    }
    const int score = (int)(keyA >> kKeyRankBits);
    const int ra = (int)(keyA & kKeyRankMask), rb = (int)(keyB & kKeyRankMask);
    const int sA = score >= total ? -L : (ra <= T ? ra : -(ra - T));
    // rank in the (C, A) order: 0 for shift 0, -s for s < 0, T + s for s > 0
    const int sB = score >= total ? -L : (rb <= T ? -rb : rb - T);
    ac = shd_from_shift(sA, score, L, L);
    ca = shd_from_shift(sB == -L ? -L : -sB, score, L, L);
}

// The alignment stage with a warp per work item (a mirrored pair or a single
// pair; the same items and outputs as k_align). Persistent: the grid's warps
// stride over the items.
template <int BLOCK, int NW, bool CNT = false>
__global__ void __launch_bounds__(BLOCK)
k_align_warp(DevOptions o, DevReads r, uint32_t first, const uint32_t* __restrict__ cand_ids,
             const uint32_t* __restrict__ cand_anchor, const uint32_t* __restrict__ seg_off,
             const uint32_t* __restrict__ seg_cnt, const unsigned long long* __restrict__ total_ptr,
             unsigned long long arena_cap, const int* __restrict__ status, AlignRes* __restrict__ out,
             unsigned long long* __restrict__ work_count, const uint32_t* __restrict__ pair_order,
             const uint2* __restrict__ work, const unsigned int* __restrict__ work_n,
             unsigned long long* __restrict__ run_count) {
    using Cnt = typename std::conditional<CNT, WordCount, NoCount>::type;
    __shared__ int s_mex[kMaxLen + 1];
    for (int i = threadIdx.x; i <= kMaxLen; i += BLOCK) s_mex[i] = __float2int_rz(__fmul_rn((float)i, o.max_error_rate));
    __syncthreads();
    if (*status & kStatusCandOverflow) return;
    const unsigned long long total = *total_ptr;
    if (total > arena_cap) return;
    const unsigned long long items = work ? (unsigned long long)work_n[0] + work_n[1] : total;
    const int lane = threadIdx.x & 31;
    const unsigned long long nwarps = (unsigned long long)gridDim.x * (BLOCK / 32);
    const float ler = __fmul_rn(o.estimated_errorrate, 4.0f);
#pragma unroll 1
    for (unsigned long long slot = (unsigned long long)blockIdx.x * (BLOCK / 32) + (threadIdx.x >> 5); slot < items;
         slot += nwarps) {
        Cnt wc;
        unsigned long long i;
        uint32_t j = kNoMirror;
        if (work) {
            const unsigned nl = work_n[0];
            const uint2 wv = slot < nl ? work[slot] : work[total - 1 - (slot - nl)];
            i = wv.x;
            j = wv.y;
        } else {
            i = pair_order ? pair_order[slot] : slot;
        }
        const uint32_t ai = cand_anchor[i];
        const uint32_t a = first + ai;
        const uint32_t c = cand_ids[i];
        const int La = r.len[a], Lc = r.len[c];
        uint32_t Ah[NW + 2], Al[NW + 2], Ch[NW + 2], Cl[NW + 2];
        load_planes<NW>(r.seq + (size_t)a * r.seq_pitch, La, Ah, Al);
        load_planes<NW>(r.seq + (size_t)c * r.seq_pitch, Lc, Ch, Cl);
        const int lo = __float2int_rz(__fmul_rn((float)La, o.min_overlap_ratio));
        const int minov = o.min_overlap > lo ? o.min_overlap : lo;
        if (work_count && lane == 0) atomicAdd(work_count, (unsigned long long)(2 * unpruned_words(La, Lc, minov)));
        ShdResult f, g;
        if (j != kNoMirror) shifted_hamming_pair_lanes<NW, Cnt>(Ah, Al, Ch, Cl, La, minov, s_mex, f, g, &wc);
        else f = shifted_hamming_lanes<NW, Cnt>(Ah, Al, La, Ch, Cl, Lc, minov, s_mex, &wc);
        uint32_t Rh[NW + 2], Rl[NW + 2];
        revcomp_planes<NW>(Ch, Cl, Lc, Rh, Rl);
        const ShdResult rc = shifted_hamming_lanes<NW, Cnt>(Ah, Al, La, Rh, Rl, Lc, minov, s_mex, &wc);
        if constexpr (CNT) {
            const unsigned ws = __reduce_add_sync(0xffffffffu, (unsigned)wc.n);
            if (lane == 0) atomicAdd(run_count, (unsigned long long)ws);
        }
        if (lane == 0) {
            auto result = [&](const ShdResult& fw, uint32_t anchor_index, uint32_t cand) {
                const int orient = choose_orientation(fw, rc, La, o.min_overlap_ratio, o.min_overlap, ler);
                AlignRes res;
                const ShdResult& b = orient == 2 ? rc : fw;
                res.shift = (int16_t)b.shift;
                res.overlap = (int16_t)b.overlap;
                res.nops = (int16_t)b.nops;
                res.orient = (uint8_t)orient;
                res.paired = o.paired_end ? mate_flag(cand_ids, seg_off, seg_cnt, anchor_index, cand) : 0;
                return res;
            };
            out[i] = result(f, ai, c);
            if (j != kNoMirror) out[j] = result(g, c - first, a);
        }
    }
}

// ---------------------------------------------------------------------------
// Stage 3: filters, MSA, refinement, correction.
//   filterCandidatesByAlignmentFlag / ...MismatchRatio(WithPairFlags)
//                                     include/corrector.hpp:982-1211
//   alignmentsComputeWeightsAndAoStoSoA :1260-1280, calculateOverlapWeight
//                                     include/hostdevicefunctions.cuh:93-97
//   MultipleSequenceAlignment::build/addSequence/findConsensus/
//   findOrigWeightAndCoverage         src/msa.cpp:9-173
//   refineMSA                         include/corrector.hpp:1307-1421
//   findCandidatesOfDifferentRegion   src/msa.cpp:532-734
//   getMSAProperties                  src/msa.cpp:304-376
//   getCorrectedAnchor                src/msa.cpp:379-453
//   getCorrectedCandidates            src/msa.cpp:457-522
//   makeOutputOfTask (edits)          include/corrector.hpp:1639-1761
//
// Layout: warp w owns the 32-column blocks w, w+NWARP, ...; lane l owns
// column 32*block + l. A column's sums are accumulated by its owner, anchor
// first and then candidates in list order, with separate IEEE multiply and
// add (no FMA) -- the reference's order and rounding, so the sums are
// bit-identical. A warp skips a candidate that covers none of a block's
// columns (a warp-uniform test). Candidate rows are staged in shared memory
// as their packed sequence and quality words (all warps loading, eight rows
// in flight per lane) and read in place; they stay staged across refinement
// rebuilds when the candidate list fits (up to 128 rows in 16 KB).
// ---------------------------------------------------------------------------
struct MsaOut {
    uint8_t* status;
    int32_t* nedits;
    char* seq;                        // count * max_len
    uint32_t* corr_id;
    uint32_t* corr_anchor;
    int32_t* corr_shift;
    uint8_t* corr_use_edits;
    char* corr_seq;                   // corr_cap * max_len
    unsigned long long* corr_count;
    unsigned long long corr_cap;
    // decision columns (EMIT): 24 features, read id, pos | orig << 16 | cons << 18
    float* feat;
    uint32_t* feat_read;
    uint32_t* feat_meta;
    unsigned long long* feat_count;
    unsigned long long feat_cap;
    // elements added to column sums (anchor and candidate bases, every
    // build): the MSA stage's roofline work; may be null
    unsigned long long* elem_count;
    // refinement statistics, may be null: [0] elements added by rebuilds
    // (builds after the first), [1] anchors rebuilt at least once
    unsigned long long* rebuild_count;
};

constexpr int kNumFeatures = 24;

constexpr int kStageMax = 128;        // candidate rows held in shared memory, at most
constexpr int kStageBudget = 16384;   // bytes of staged rows
constexpr int kStageGuard = 32;       // bytes before and after the staged rows

// words of a staged row (qb: the quality encoding the sums read). The bases
// are realigned to the anchor's 16-base grid, so they take one word more than
// the read's pitch; 1- and 8-bit quality codes follow on their own grids (32
// and 4 codes per word), 2-bit codes are interleaved with the bases as word
// pairs {bases, qualities} of the same 16 positions.
__host__ __device__ inline int msa_slot_words(int seq_pitch, int qual_pitch, int qb) {
    if (qb == 0) return seq_pitch + 1;
    if (qb == 2) return 2 * ((seq_pitch > qual_pitch ? seq_pitch : qual_pitch) + 1);
    return seq_pitch + 1 + qual_pitch + 1;
}

// candidate rows staged at once
__host__ __device__ inline int msa_stage_rows(int seq_pitch, int qual_pitch, int qb) {
    const int rows = kStageBudget / (msa_slot_words(seq_pitch, qual_pitch, qb) * 4);
    return rows > kStageMax ? kStageMax : (rows < 16 ? 16 : rows);
}

// dynamic shared memory of k_msa: the anchor's decoded row, the staged
// candidate rows (between two guard bands: a lane whose column lies outside
// a row may read a few words past either end of it, and adds nothing); with
// decision rows also three per-anchor-column weights; then the per-column
// arrays of `maxcols` columns (four 16-bit counts, support, coverage,
// consensus). Every part starts on a 16-byte boundary (maxcols is a multiple
// of 128).
__host__ __device__ inline size_t msa_round16(size_t x) { return (x + 15) & ~(size_t)15; }
__host__ __device__ inline size_t msa_raw_bytes(int seq_pitch, int qual_pitch, int qb) {
    return msa_round16(2 * kStageGuard + (size_t)msa_stage_rows(seq_pitch, qual_pitch, qb) *
                                             msa_slot_words(seq_pitch, qual_pitch, qb) * 4);
}
__host__ __device__ inline size_t msa_smem_bytes(int max_len, int seq_pitch, int qual_pitch, int qb, bool emit,
                                                 int maxcols) {
    const size_t elem = msa_round16((size_t)max_len * 2);
    const size_t fw = emit ? msa_round16((size_t)3 * max_len * 4) : 0;
    return elem + msa_raw_bytes(seq_pitch, qual_pitch, qb) + fw + (size_t)maxcols * (8 + 4 + 2 + 1);
}

// Realigned and reversed rows: a window of one word of codes whose first
// code is code s0 of a source row (codes before the row and past its end
// read as zero), the source row's words held one per lane in m (zero from
// the row's pitch on; lane 31 zero for the 2- and 1-bit forms, whose pitches
// are at most 16 and 8 words). Branch free: the row is read as if preceded
// by one zero word, and a funnel shift with a zero count returns its high
// word.
// 2-bit codes, 16 per word, MSB first
__device__ __forceinline__ uint32_t window2(uint32_t m, int s0) {
    const int sc = max(s0 + 16, 0);
    const int wi = sc >> 4;
    const uint32_t a = __shfl_sync(0xffffffffu, m, (wi + 31) & 31);    // source word wi - 1
    const uint32_t b = __shfl_sync(0xffffffffu, m, wi & 31);
    return __funnelshift_l(b, a, 2 * (sc & 15));
}
// 1-bit codes, 32 per word, MSB first
__device__ __forceinline__ uint32_t window1(uint32_t m, int s0) {
    const int sc = max(s0 + 32, 0);
    const int wi = sc >> 5;
    const uint32_t a = __shfl_sync(0xffffffffu, m, (wi + 31) & 31);
    const uint32_t b = __shfl_sync(0xffffffffu, m, wi & 31);
    return __funnelshift_l(b, a, sc & 31);
}
// 8-bit codes, 4 per word, little-endian; source words 0..31 in m0, 32..63 in m1
__device__ __forceinline__ uint32_t window8(uint32_t m0, uint32_t m1, int s0) {
    const int sc = max(s0 + 4, 0);
    const int wi = sc >> 2;
    const int ia = wi - 1, ib = wi;
    const uint32_t a0 = __shfl_sync(0xffffffffu, m0, ia & 31), a1 = __shfl_sync(0xffffffffu, m1, ia & 31);
    const uint32_t b0 = __shfl_sync(0xffffffffu, m0, ib & 31), b1 = __shfl_sync(0xffffffffu, m1, ib & 31);
    const uint32_t a = ia < 0 ? 0u : ia < 32 ? a0 : a1;
    const uint32_t b = ib < 32 ? b0 : b1;
    return __funnelshift_r(a, b, 8 * (sc & 3));
}
// reverse the 16 2-bit codes of a word, keeping each code's bits
__device__ __forceinline__ uint32_t rev2(uint32_t w) {
    w = __brev(w);
    return ((w >> 1) & 0x55555555u) | ((w & 0x55555555u) << 1);
}

// One element of a column: weight w added to the sum of its base (b8 = base
// * 8) and one to the base's 8-bit count in c8 (A | C << 8 | G << 16 |
// T << 24), nothing when the column lies outside the row (p, the column's
// position in the row, not below len). IEEE adds (add.rn.f32, no
// contraction), predicated on (base, in row): the sums see the same
// additions in the same order as an add per element of the base.
__device__ __forceinline__ void msa_add8(float& wA, float& wC, float& wG, float& wT, uint32_t& c8,
                                         uint32_t b8, float w, int p, int len) {
    asm("{\n\t"
        ".reg .pred pin, pa, pc, pg, pt;\n\t"
        ".reg .b32 inc;\n\t"
        "setp.lt.u32 pin, %7, %8;\n\t"
        "setp.eq.and.b32 pa, %6, 0, pin;\n\t"
        "setp.eq.and.b32 pc, %6, 8, pin;\n\t"
        "setp.eq.and.b32 pg, %6, 16, pin;\n\t"
        "setp.eq.and.b32 pt, %6, 24, pin;\n\t"
        "@pa add.rn.f32 %0, %0, %5;\n\t"
        "@pc add.rn.f32 %1, %1, %5;\n\t"
        "@pg add.rn.f32 %2, %2, %5;\n\t"
        "@pt add.rn.f32 %3, %3, %5;\n\t"
        "shl.b32 inc, %9, %6;\n\t"
        "@pin add.u32 %4, %4, inc;\n\t"
        "}"
        : "+f"(wA), "+f"(wC), "+f"(wG), "+f"(wT), "+r"(c8)
        : "f"(w), "r"(b8), "r"(p), "r"(len), "r"(1u));
}

// The whole MSA stage of one anchor (local index ai) for one CTA. Every
// early return is taken by all threads of the CTA together.
// QB: the quality encoding the sums read (0: qualities unused, else 1, 2 or
// 8 bits per quality); jb: 32-column blocks per warp (the MSA holds at most
// 32 * jb * warps columns).
template <int BLOCK, int QB, bool EMIT>
__device__ __forceinline__ void
msa_anchor(const DevOptions& o, const DevReads& r, uint32_t first, uint32_t ai, int jb,
           const uint32_t* __restrict__ cand_ids, const uint32_t* __restrict__ seg_off,
           const uint32_t* __restrict__ seg_cnt, const AlignRes* __restrict__ ares,
           CandRec* __restrict__ recs, const MsaOut& out, int* __restrict__ status) {
    constexpr int NWARP = BLOCK / 32;
    const int MAXCOLS = 32 * jb * NWARP;
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ float s_qw[256];
    // per warp: the staged rows meeting its column block, {row grid offset,
    // first position - lane, length, weights}, and for 1- and 8-bit qualities
    // the row's quality grid offset
    __shared__ uint4 s_hits[NWARP][33];
    __shared__ int s_hq[(QB == 1 || QB == 8) ? NWARP : 1][33];
    __shared__ int s_blk;                    // next column block (persistent rows: warps take blocks in turn)
    __shared__ float s_qwc[4];               // weight of a 1- or 2-bit quality code
    __shared__ int s_beg[kStageMax], s_len[kStageMax];
    __shared__ float s_w[kStageMax];
    __shared__ uint32_t s_id[kStageMax];
    __shared__ uint8_t s_fwd[kStageMax];
    __shared__ int2 s_bl[kStageMax];         // {begin, length} of staged row k
    __shared__ float s_wq[kStageMax][4];     // row weight * weight of a 1- or 2-bit quality code
    __shared__ uint8_t s_alive[kStageMax];
    __shared__ int s_red[NWARP][4];
    __shared__ int s_vals[12];
    __shared__ uint16_t s_dec[EMIT ? kMaxLen : 1];   // decision positions of the anchor (EMIT)
    __shared__ __align__(16) float s_asup[kMaxLen];   // support of the anchor's columns, position order

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t a = first + ai;
    const uint32_t off = seg_off[ai], cnt = seg_cnt[ai];
    const int La = r.len[a];
    const int mlen = r.max_len;
    constexpr bool useQ = QB != 0;
    char* aout = out.seq + (size_t)ai * mlen;
    const int nstage = msa_stage_rows(r.seq_pitch, r.qual_pitch, QB);
    const int rw = msa_slot_words(r.seq_pitch, r.qual_pitch, QB);   // words per staged row
    // dynamic shared memory, each part 16-byte aligned (msa_smem_bytes)
    uint16_t* s_aelem = (uint16_t*)dsm;                      // anchor row: base | quality char << 2
    unsigned char* s_rawg = dsm + msa_round16((size_t)mlen * 2);
    uint32_t* s_raw = (uint32_t*)(s_rawg + kStageGuard);     // [nstage][rw]
    // per anchor column: column weight sum, consensus weight, weight of the
    // anchor's base (EMIT only)
    float* s_fw = (float*)(s_rawg + msa_raw_bytes(r.seq_pitch, r.qual_pitch, QB));
    // per MSA column: counts of A C G T, support, coverage, consensus
    ushort4* s_cnt4 = (ushort4*)((unsigned char*)s_fw + (EMIT ? msa_round16((size_t)3 * mlen * 4) : 0));
    float* s_support = (float*)(s_cnt4 + MAXCOLS);
    uint16_t* s_cov = (uint16_t*)(s_support + MAXCOLS);
    uint8_t* s_cons = (uint8_t*)(s_cov + MAXCOLS);
    auto cnt_of = [&](int col, int b) -> int {
        const ushort4 c = s_cnt4[col];
        return b == 0 ? c.x : b == 1 ? c.y : b == 2 ? c.z : c.w;
    };

    if (cnt == 0) {
        if (tid == 0) { out.status[ai] = 0; out.nedits[ai] = 0; }
        return;
    }

    auto block_sum4 = [&](int v0, int v1, int v2, int v3, int* res) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            v0 += __shfl_xor_sync(0xffffffffu, v0, d);
            v1 += __shfl_xor_sync(0xffffffffu, v1, d);
            v2 += __shfl_xor_sync(0xffffffffu, v2, d);
            v3 += __shfl_xor_sync(0xffffffffu, v3, d);
        }
        __syncthreads();
        if (lane == 0) { s_red[warp][0] = v0; s_red[warp][1] = v1; s_red[warp][2] = v2; s_red[warp][3] = v3; }
        __syncthreads();
        int t0 = 0, t1 = 0, t2 = 0, t3 = 0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) { t0 += s_red[w][0]; t1 += s_red[w][1]; t2 += s_red[w][2]; t3 += s_red[w][3]; }
        res[0] = t0; res[1] = t1; res[2] = t2; res[3] = t3;
    };
    // block-wide exclusive scan of one value per thread; *tot gets the sum
    auto block_scan = [&](int v, int* tot) {
        int x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        __syncthreads();
        if (lane == 31) s_red[warp][0] = x;
        __syncthreads();
        int pre = 0, all = 0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) { const int sv = s_red[w][0]; if (w < warp) pre += sv; all += sv; }
        *tot = all;
        return pre + x - v;
    };

    // ---- quality weights (qualityscoreweights.hpp:12-44) ----
    for (int i = tid; i < 256; i += BLOCK) s_qw[i] = c_qweight[i];
    constexpr int qbits = QB;
    if (tid < 4) {
        // the characters a 2- or 1-bit code stands for (qualityscorecompression.hpp:121-145)
        const uint32_t ch = qbits == 2 ? (tid == 0 ? '$' : tid == 1 ? '(' : tid == 2 ? '1' : '9')
                                       : (tid == 1 ? '5' : '(');
        s_qwc[tid] = c_qweight[ch];
    }

    // ---- alignment filters (corrector.hpp:982-1211), ordered compaction ----
    const float base = fmul_rn(o.estimated_errorrate, 1.0f);
    const float base2 = fmul_rn(2.0f, base), base3 = fmul_rn(3.0f, base), base4 = fmul_rn(4.0f, base);
    int c0 = 0, c1 = 0, c2 = 0, n1 = 0;
    // the first candidate of each thread: its alignment, mismatch ratio, id
    // and length stay in registers for the compaction below (the id and
    // length loads overlap the counting)
    AlignRes ar0{};
    float mr0 = 0.0f;
    uint32_t id0 = 0;
    int len0 = 0;
    for (uint32_t i = tid; i < cnt; i += BLOCK) {
        const AlignRes ar = ares[off + i];
        float mr = 0.0f;
        if (ar.orient != 3) {
            n1++;
            mr = fdiv_rn((float)ar.nops, (float)ar.overlap);
            c0 += mr < base2;
            c1 += mr < base3;
            c2 += mr < base4;
        }
        if (i == (uint32_t)tid) {
            ar0 = ar;
            mr0 = mr;
            id0 = cand_ids[off + i];
            len0 = r.len[id0];
        }
    }
    int red[4];
    block_sum4(c0, c1, c2, n1, red);
    if (red[3] == 0) {
        if (tid == 0) { out.status[ai] = 0; out.nedits[ai] = 0; }
        return;
    }
    float thr = -3.402823466e+38f;
    {
        const float good = fmul_rn(o.estimated_coverage, o.m_coverage);
        if (red[0] > 0 || red[1] > 0 || red[2] > 0) {
            if ((float)red[0] >= good) thr = base2;
            else if ((float)red[1] >= good) thr = base3;
            else if ((float)red[2] >= good) thr = base4;
        }
    }
    // every candidate fits the staged rows: the survivors' records go straight
    // to shared memory (else to the global records, staged chunk by chunk)
    const bool direct = cnt <= (uint32_t)nstage;
    int V = 0;
    for (uint32_t c = 0; c < cnt; c += BLOCK) {
        const uint32_t i = c + tid;
        int keep = 0;
        AlignRes ar = ar0;
        float mr = mr0;
        if (i < cnt) {
            if (c) {
                ar = ares[off + i];
                if (ar.orient != 3) mr = fdiv_rn((float)ar.nops, (float)ar.overlap);
            }
            if (ar.orient != 3)
                keep = o.paired_end ? (ar.paired || mr < o.paired_filter_threshold) : (mr < thr);
        }
        int tot;
        const int pre = block_scan(keep, &tot);
        if (keep) {
            CandRec rec;
            rec.id = c ? cand_ids[off + i] : id0;
            rec.shift = ar.shift;
            rec.len = (uint16_t)(c ? r.len[rec.id] : len0);
            // calculateOverlapWeight: 1 - sqrtf(nOps / (overlap * maxMismatchRatio))
            rec.weight = fsub_rn(1.0f, __fsqrt_rn(fdiv_rn((float)ar.nops, fmul_rn((float)ar.overlap, o.max_error_rate))));
            rec.orient = ar.orient;
            const int k = V + pre;
            if (direct) {
                s_beg[k] = rec.shift;
                s_len[k] = rec.len;
                s_w[k] = rec.weight;
                s_fwd[k] = rec.orient == 1;
                s_id[k] = rec.id;
                s_bl[k] = make_int2(rec.shift, rec.len);
#pragma unroll
                for (int q = 0; q < 4; ++q) s_wq[k][q] = fmul_rn(rec.weight, s_qwc[q]);
            } else {
                recs[off + k] = rec;
            }
        }
        V += tot;
    }
    if (V == 0) {
        if (tid == 0) { out.status[ai] = 0; out.nedits[ai] = 0; }
        return;
    }
    __syncthreads();

    // ---- anchor row ----
    const int sp = r.seq_pitch, qp = r.qual_pitch;
    // quality character at position q of an encoded row (qualityscorecompression.hpp:121-145)
    auto qual_char = [&](const uint32_t* row, int q) -> uint32_t {
        if (qbits == 8) return (row[q >> 2] >> (8 * (q & 3))) & 0xFFu;
        if (qbits == 2) {
            const uint32_t b = (row[q >> 4] >> (30 - 2 * (q & 15))) & 3u;
            return b == 0 ? '$' : b == 1 ? '(' : b == 2 ? '1' : '9';
        }
        return ((row[q >> 5] >> (31 - (q & 31))) & 1u) ? '5' : '(';
    };
    {
        const uint32_t* arow = r.seq + (size_t)a * sp;
        const uint32_t* aq = useQ ? r.qual + (size_t)a * qp : nullptr;
        for (int p = tid; p < La; p += BLOCK) {
            const uint32_t b = base_at(arow, p);
            const uint32_t q = useQ ? qual_char(aq, p) : 0u;
            s_aelem[p] = (uint16_t)(b | (q << 2));
        }
    }

    // stage candidate rows [c, c+n) of recs into slots 0..n-1, realigned to
    // the anchor's grid: the code at row position p of a row with shift s
    // moves to anchor-relative position s + p, which lies in word
    // (s + p) / 16 - s / 16 of the row's bases (floor divisions; 32 and 4
    // codes per word for 1- and 8-bit qualities). Reverse-complement rows are
    // turned into the alignment's orientation on the way (bases reversed and
    // complemented, qualities reversed over the whole quality pitch:
    // reverseQualitiesOfRCAlignments, corrector.hpp:1227-1239), so the column
    // sums read every row forward, and a lane finds its column's code at the
    // same bits of every row. A warp per row: lane j loads word j of the
    // row's packed bases and of its quality words (RR rows of a warp in
    // flight: two measured best, 21.6 ms per 1M anchors against 22.1 ms with
    // one and 22.3 ms with four), then builds output word j from a window of
    // them.
    auto stage = [&](int c, int n, bool fill, auto RR) {
        constexpr int R = decltype(RR)::value;
        __syncthreads();
        if (fill) {
            for (int k = tid; k < n; k += BLOCK) {
                const CandRec rc = recs[off + c + k];
                s_beg[k] = rc.shift;                // relative to the anchor; abegin added per build
                s_len[k] = rc.len;
                s_w[k] = rc.weight;
                s_fwd[k] = rc.orient == 1;
                s_id[k] = rc.id;
                s_bl[k] = make_int2(rc.shift, rc.len);
#pragma unroll
                for (int q = 0; q < 4; ++q) s_wq[k][q] = fmul_rn(rc.weight, s_qwc[q]);
            }
            __syncthreads();
        }
        for (int k0 = warp * R; k0 < n; k0 += NWARP * R) {
            uint32_t ms[R], mq0[R], mq1[R];
#pragma unroll
            for (int t = 0; t < R; ++t) {
                ms[t] = mq0[t] = mq1[t] = 0u;
                if (k0 + t < n) {
                    const size_t id = s_id[k0 + t];
                    if (lane < sp) ms[t] = __ldg(r.seq + id * sp + lane);
                    if constexpr (useQ) {
                        const uint32_t* qrow = r.qual + id * qp;
                        if (lane < qp) mq0[t] = __ldg(qrow + lane);
                        if constexpr (QB == 8) if (lane + 32 < qp) mq1[t] = __ldg(qrow + lane + 32);
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int k = k0 + t;
                if (k >= n) break;                           // warp-uniform
                uint32_t* row = s_raw + k * rw;
                const bool rev = !s_fwd[k];                  // warp-uniform
                const int L = s_len[k], sft = s_beg[k];
                const int o16 = sft & 15;
                uint32_t ws = window2(ms[t], rev ? L - 16 - 16 * lane + o16 : 16 * lane - o16);
                if (rev) ws = ~rev2(ws);                     // reversed, complemented: A<->T, C<->G
                if constexpr (QB == 2) {
                    uint32_t wq = window2(mq0[t], rev ? mlen - 16 - 16 * lane + o16 : 16 * lane - o16);
                    if (rev) wq = rev2(wq);
                    if (lane <= (sp > qp ? sp : qp)) reinterpret_cast<uint2*>(row)[lane] = make_uint2(ws, wq);
                } else {
                    if (lane <= sp) row[lane] = ws;
                    if constexpr (QB == 1) {
                        const int o32 = sft & 31;
                        uint32_t wq = window1(mq0[t], rev ? mlen - 32 - 32 * lane + o32 : 32 * lane - o32);
                        if (rev) wq = __brev(wq);
                        if (lane <= qp) row[sp + 1 + lane] = wq;
                    } else if constexpr (QB == 8) {
                        const int o4 = sft & 3;
#pragma unroll
                        for (int h = 0; h < 3; ++h) {
                            const int j = lane + 32 * h;
                            uint32_t wq = window8(mq0[t], mq1[t], rev ? mlen - 4 - 4 * j + o4 : 4 * j - o4);
                            if (rev) wq = __byte_perm(wq, 0u, 0x0123);
                            if (j <= qp) row[sp + 1 + j] = wq;
                        }
                    }
                }
            }
        }
        __syncthreads();
    };
    // base (2-bit, in the candidate's aligned orientation) of staged row k at
    // position p < s_len[k]
    auto cand_base = [&](int k, int p) -> uint32_t {
        const int sft = s_beg[k], q = sft + p;
        const int wi = (q >> 4) - (sft >> 4);
        const uint32_t w = s_raw[k * rw + (QB == 2 ? 2 * wi : wi)];
        return (w >> (30 - 2 * (q & 15))) & 3u;
    };
    const bool persistent = V <= nstage;      // all rows stay staged across rebuilds
    int nalive = V;
    if (persistent) {
        stage(0, V, !direct, std::integral_constant<int, 2>{});
        for (int k = tid; k < V; k += BLOCK) s_alive[k] = (uint8_t)k;
    }
    __syncthreads();

    int abegin = 0, aend = 0, ncols = 0;
    bool allGood = false, hq = false;

    for (int iter = 0;; ++iter) {
        // ---- MSA geometry (build, msa.cpp:17-33) ----
        int mn = 0, mx = La, sl = 0;                // sl: bases of the rows (roofline work)
        if (persistent) {
            for (int i = tid; i < nalive; i += BLOCK) {
                const int k = s_alive[i];
                mn = min(mn, s_beg[k]);
                mx = max(mx, s_beg[k] + s_len[k]);
                sl += s_len[k];
            }
        } else {
            for (int k = tid; k < nalive; k += BLOCK) {
                const CandRec rc = recs[off + k];
                mn = min(mn, (int)rc.shift);
                mx = max(mx, (int)rc.shift + (int)rc.len);
                sl += rc.len;
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, d));
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
            sl += __shfl_xor_sync(0xffffffffu, sl, d);
        }
        if (tid == 0) s_blk = 0;             // the previous build's sums are done (CTA barrier after them)
        __syncthreads();
        if (lane == 0) { s_red[warp][0] = mn; s_red[warp][1] = mx; s_red[warp][2] = sl; }
        __syncthreads();
        mn = 0; mx = La;
        for (int w = 0; w < NWARP; ++w) { mn = min(mn, s_red[w][0]); mx = max(mx, s_red[w][1]); }
        if (tid == 0 && out.elem_count) {
            int tot = La;
            for (int w = 0; w < NWARP; ++w) tot += s_red[w][2];
            atomicAdd(out.elem_count, (unsigned long long)tot);
            if (iter > 0 && out.rebuild_count) {
                atomicAdd(out.rebuild_count, (unsigned long long)tot);
                if (iter == 1) atomicAdd(out.rebuild_count + 1, 1ull);
            }
        }
        ncols = mx - mn;
        abegin = -mn;
        aend = abegin + La;
        if (ncols > MAXCOLS) {
            if (tid == 0) { atomicOr(status, kStatusColumns); out.status[ai] = 0; out.nedits[ai] = 0; }
            return;
        }

        // ---- column sums (anchor first, then candidates in list order) and
        //      consensus (findConsensus, msa.cpp:135-157): each warp takes one
        //      32-column block at a time, lane = column ----
        // persistent rows: the warps take the column blocks in turn from a
        // shared counter (blocks differ in their row counts); rows staged in
        // chunks: every warp runs its jb blocks (staging synchronises the CTA)
        const int nblk = (ncols + 31) >> 5;
#pragma unroll 1
        for (int j = 0;; ++j) {
            int blk;
            if (persistent) {
                if (lane == 0) blk = atomicAdd(&s_blk, 1);
                blk = __shfl_sync(0xffffffffu, blk, 0);
                if (blk >= nblk) break;
            } else {
                if (j >= jb) break;
                blk = warp + NWARP * j;
            }
            const int c0 = 32 * blk;
            const int col = c0 + lane;
            const bool active = c0 < ncols;                  // warp-uniform
            uint32_t cAC = 0u, cGT = 0u;                     // 16-bit counts: A | C << 16, G | T << 16
            uint32_t c8 = 0u;           // the chunk's 8-bit counts A | C << 8 | G << 16 | T << 24
            float wA = 0.0f, wC = 0.0f, wG = 0.0f, wT = 0.0f;
            // a chunk adds at most 128 rows and the anchor: its 8-bit counts
            // cannot overflow before they are moved to the 16-bit ones
            auto flush = [&]() {
                cAC += (c8 & 0xFFu) | ((c8 & 0xFF00u) << 8);
                cGT += ((c8 >> 16) & 0xFFu) | ((c8 >> 24) << 16);
                c8 = 0u;
            };
            {
                const int p = col - abegin;
                if (active && p >= 0 && p < La) {
                    const uint32_t e = s_aelem[p];
                    msa_add8(wA, wC, wG, wT, c8, (e & 3u) << 3, useQ ? s_qw[e >> 2] : 1.0f, 0, 1);   // factor 1.0f
                }
            }
            // staged rows (slot list[i], or slot i) meeting this block, in
            // list order: per chunk of 32 rows the warp lists the rows that
            // meet the block (ballot, order kept) as {grid origin of the row
            // in bytes, first position - lane, length, weights}; two listed
            // rows load together, then add in order (measured: 21.6 ms per
            // 1M anchors against 22.3 ms with four and 24.3 ms with one). The
            // last listed row is repeated past the list with length 0: a pair
            // reads it there, in bounds, and adds nothing.
            auto run_rows = [&](const uint8_t* list, int nrows) {
                // this lane's column on the anchor's grid: the word of every
                // staged row that holds it (byte offset, relative to the
                // row's grid origin) and its bits there, as rotations that
                // bring the base to bits 3-4 (base * 8) and the quality code
                // to bits 2-3 (2-bit) or bit 2 (1-bit), i.e. the byte offset
                // of its weight
                const int q = col - abegin;
                const int qsh = 30 - 2 * (q & 15);
                const uint32_t rb8 = (uint32_t)(qsh + 29) & 31u;
                const int loff = (q >> 4) * (QB == 2 ? 8 : 4);
                uint32_t rq = 0u;
                int qoff = 0;
                if constexpr (QB == 2) rq = (uint32_t)(qsh + 30) & 31u;
                if constexpr (QB == 1) { rq = (uint32_t)(31 - (q & 31) + 30) & 31u; qoff = (q >> 5) * 4; }
                if constexpr (QB == 8) { rq = 8u * (uint32_t)(q & 3); qoff = (q >> 2) * 4; }
                const unsigned char* rawb = reinterpret_cast<const unsigned char*>(s_raw);
                const unsigned char* wqb = reinterpret_cast<const unsigned char*>(&s_wq[0][0]);
                for (int i0 = 0; i0 < nrows; i0 += 32) {
                    bool hit = false;
                    uint4 ent = make_uint4(0u, 0u, 0u, 0u);
                    int hq = 0;
                    if (i0 + lane < nrows) {
                        const int k = list ? list[i0 + lane] : i0 + lane;
                        const int2 bl = s_bl[k];
                        const int cb = abegin + bl.x;
                        hit = cb < c0 + 32 && cb + bl.y > c0;
                        ent.x = (uint32_t)(k * rw * 4 - (bl.x >> 4) * (QB == 2 ? 8 : 4));
                        ent.y = (uint32_t)(c0 - cb);
                        ent.z = (uint32_t)bl.y;
                        ent.w = (QB == 1 || QB == 2) ? (uint32_t)k * 16u : __float_as_uint(s_w[k]);
                        if constexpr (QB == 1) hq = (k * rw + sp + 1 - (bl.x >> 5)) * 4;
                        if constexpr (QB == 8) hq = (k * rw + sp + 1 - (bl.x >> 2)) * 4;
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    const int nh = __popc(m);
                    if (hit) {
                        const int pos = __popc(m & ((1u << lane) - 1u));
                        s_hits[warp][pos] = ent;
                        if constexpr (QB == 1 || QB == 8) s_hq[warp][pos] = hq;
                        if (pos == nh - 1) {
                            s_hits[warp][pos + 1] = make_uint4(ent.x, ent.y, 0u, ent.w);
                            if constexpr (QB == 1 || QB == 8) s_hq[warp][pos + 1] = hq;
                        }
                    }
                    __syncwarp();
                    for (int h0 = 0; h0 < nh; h0 += 2) {
                        uint32_t bb[2];
                        float ww[2];
                        int pp[2], ll[2];
#pragma unroll
                        for (int u = 0; u < 2; ++u) {
                            const uint4 e = s_hits[warp][h0 + u];
                            const unsigned char* wp = rawb + ((int)e.x + loff);
                            uint32_t sw, qv = 0u;
                            if constexpr (QB == 2) {
                                const uint2 t2 = *reinterpret_cast<const uint2*>(wp);
                                sw = t2.x;
                                qv = t2.y;
                            } else {
                                sw = *reinterpret_cast<const uint32_t*>(wp);
                                if constexpr (QB == 1 || QB == 8)
                                    qv = *reinterpret_cast<const uint32_t*>(rawb + (s_hq[warp][h0 + u] + qoff));
                            }
                            bb[u] = __funnelshift_r(sw, sw, rb8) & 24u;
                            if constexpr (QB == 0) ww[u] = __uint_as_float(e.w);
                            else if constexpr (QB == 2)
                                ww[u] = *reinterpret_cast<const float*>(wqb + (e.w + (__funnelshift_r(qv, qv, rq) & 12u)));
                            else if constexpr (QB == 1)
                                ww[u] = *reinterpret_cast<const float*>(wqb + (e.w + (__funnelshift_r(qv, qv, rq) & 4u)));
                            else ww[u] = fmul_rn(__uint_as_float(e.w), s_qw[(qv >> rq) & 0xFFu]);
                            pp[u] = lane + (int)e.y;
                            ll[u] = (int)e.z;
                        }
#pragma unroll
                        for (int u = 0; u < 2; ++u) msa_add8(wA, wC, wG, wT, c8, bb[u], ww[u], pp[u], ll[u]);
                    }
                    __syncwarp();
                }
            };
            // persistent rows are one chunk; with more rows than fit, each
            // chunk is staged (by all warps) per block
            const int nchunk = persistent ? 1 : (nalive + nstage - 1) / nstage;
            for (int ch = 0; ch < nchunk; ++ch) {
                int n = nalive;
                if (!persistent) {
                    n = min(nstage, nalive - ch * nstage);
                    stage(ch * nstage, n, true, std::integral_constant<int, 1>{});
                }
                if (active) run_rows(persistent ? s_alive : nullptr, n);
                flush();
            }
            if (active && col < ncols) {
                uint8_t cs = 0; float cw = wA;
                if (wC > cw) { cs = 1; cw = wC; }
                if (wG > cw) { cs = 2; cw = wG; }
                if (wT > cw) { cs = 3; cw = wT; }
                const float colw = __fadd_rn(__fadd_rn(__fadd_rn(wA, wC), wG), wT);
                s_cons[col] = cs;
                const float sup = fdiv_rn(cw, colw);
                s_support[col] = sup;
                {
                    const int p = col - abegin;
                    if (p >= 0 && p < La) s_asup[p] = sup;
                }
                const uint32_t nA = cAC & 0xFFFFu, nC = cAC >> 16;
                const uint32_t nG = cGT & 0xFFFFu, nT = cGT >> 16;
                s_cov[col] = (uint16_t)(nA + nC + nG + nT);
                s_cnt4[col] = make_ushort4((uint16_t)nA, (uint16_t)nC, (uint16_t)nG, (uint16_t)nT);
                if constexpr (EMIT) {
                    const int p = col - abegin;
                    if (p >= 0 && p < La) {
                        const uint32_t ob = s_aelem[p] & 3u;
                        s_fw[p] = colw;
                        s_fw[mlen + p] = cw;
                        s_fw[2 * mlen + p] = ob == 0 ? wA : ob == 1 ? wC : ob == 2 ? wG : wT;
                    }
                }
            }
        }
        __syncthreads();

        if (iter >= 5) break;
        // ---- refinement: findCandidatesOfDifferentRegion (msa.cpp:532-734) ----
        if (tid == 0) s_vals[1] = 0x7fffffff;
        int mism = 0;
        for (int p = tid; p < La; p += BLOCK) mism |= (s_aelem[p] & 3u) != s_cons[abegin + p];
        if (__syncthreads_or(mism) == 0) break;
        const int sigThr = f2i_rz(fmul_rn((float)o.coverage_int, 0.3f));
        for (int p = tid; p < La; p += BLOCK) {
            const int col = abegin + p;
            const int cs = s_cons[col];
            bool sig = false;
#pragma unroll
            for (int b = 0; b < 4; ++b) sig |= (b != cs && sigThr <= cnt_of(col, b));
            if (sig) atomicMin(&s_vals[1], col);
        }
        __syncthreads();
        const int col = s_vals[1];
        if (col == 0x7fffffff) break;
        int foundBase = -1;                   // the last qualifying base index wins (:591-601)
        {
            const int cs = s_cons[col];
            for (int b = 0; b < 4; ++b) if (b != cs && sigThr <= cnt_of(col, b)) foundBase = b;
        }
        const int orig = s_aelem[col - abegin] & 3u;
        const bool keepMatching = orig == foundBase;
        // per candidate: remove? (discard_rows :622-665); veto by weight >= 0.90 (:672-689)
        auto removes = [&](int b) { return keepMatching ? (b != foundBase) : (b == foundBase); };
        int nrem = 0, veto = 0;
        if (persistent) {
            for (int i = tid; i < nalive; i += BLOCK) {
                const int k = s_alive[i];
                const int rb = abegin + s_beg[k], re = rb + s_len[k];
                const int rem = (col >= rb && col < re) ? removes((int)cand_base(k, col - rb)) : 0;
                nrem += rem;
                veto |= rem && s_w[k] >= 0.90f;
            }
        } else {
            for (int k = tid; k < nalive; k += BLOCK) {
                const CandRec rc = recs[off + k];
                const int rb = abegin + rc.shift, re = rb + rc.len;
                int rem = 0;
                if (col >= rb && col < re) {
                    const int p = col - rb;
                    const uint32_t* row = r.seq + (size_t)rc.id * sp;
                    rem = removes(rc.orient == 1 ? (int)base_at(row, p) : (int)(base_at(row, rc.len - 1 - p) ^ 3u));
                }
                nrem += rem;
                veto |= rem && rc.weight >= 0.90f;
            }
        }
        const int anyVeto = __syncthreads_or(veto);
        const int anyRem = __syncthreads_or(nrem);
        if (anyVeto || !anyRem) break;        // nothing removed: the rebuilt MSA would be identical
        // ordered compaction of the survivors
        int newV = 0;
        for (int c = 0; c < nalive; c += BLOCK) {
            const int i = c + tid;
            int keep = 0, k = 0;
            CandRec rc;
            if (i < nalive) {
                if (persistent) {
                    k = s_alive[i];
                    const int rb = abegin + s_beg[k], re = rb + s_len[k];
                    keep = !((col >= rb && col < re) && removes((int)cand_base(k, col - rb)));
                } else {
                    rc = recs[off + i];
                    const int rb = abegin + rc.shift, re = rb + rc.len;
                    keep = 1;
                    if (col >= rb && col < re) {
                        const int p = col - rb;
                        const uint32_t* row = r.seq + (size_t)rc.id * sp;
                        keep = !removes(rc.orient == 1 ? (int)base_at(row, p) : (int)(base_at(row, rc.len - 1 - p) ^ 3u));
                    }
                }
            }
            int tot;
            const int pre = block_scan(keep, &tot);
            __syncthreads();
            if (keep) {
                if (persistent) s_alive[newV + pre] = (uint8_t)k;
                else recs[off + newV + pre] = rc;
            }
            newV += tot;
            __syncthreads();
        }
        nalive = newV;
        __syncthreads();
    }
    V = nalive;

    // ---- MSA properties (getMSAProperties, msa.cpp:304-376) ----
    {
        float mnS = 3.402823466e+38f;
        int mnC = 0x7fffffff;
        for (int p = tid; p < La; p += BLOCK) {
            mnS = fminf(mnS, s_support[abegin + p]);
            mnC = min(mnC, (int)s_cov[abegin + p]);
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            mnS = fminf(mnS, __shfl_xor_sync(0xffffffffu, mnS, d));
            mnC = min(mnC, __shfl_xor_sync(0xffffffffu, mnC, d));
        }
        __syncthreads();
        if (lane == 0) { s_red[warp][0] = __float_as_int(mnS); s_red[warp][1] = mnC; }
        __syncthreads();
        if (warp == 0) {
            float minSup = 3.402823466e+38f;
            int minCov = 0x7fffffff;
            for (int w = 0; w < NWARP; ++w) { minSup = fminf(minSup, __int_as_float(s_red[w][0])); minCov = min(minCov, s_red[w][1]); }
            // std::accumulate order: one serial chain of IEEE adds (lane 0),
            // the supports read four at a time
            float sum = 0.0f;
            if (lane == 0) {
                const float4* v4 = reinterpret_cast<const float4*>(s_asup);
                int p = 0;
                for (; p + 4 <= La; p += 4) {
                    const float4 v = v4[p >> 2];
                    sum = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(sum, v.x), v.y), v.z), v.w);
                }
                for (; p < La; ++p) sum = __fadd_rn(sum, s_asup[p]);
            }
            sum = __shfl_sync(0xffffffffu, sum, 0);
            const float avgSup = fdiv_rn(sum, (float)La);
            const float e = o.estimated_errorrate;
            const float avgThr = fsub_rn(1.0f, fmul_rn(1.0f, e));
            const float minThr = fsub_rn(1.0f, fmul_rn(3.0f, e));
            const float covThr = fmul_rn(fdiv_rn(o.m_coverage, 6.0f), o.estimated_coverage);
            const bool good = fgeq(avgSup, avgThr) && fgeq(minSup, minThr) && fgeq((float)minCov, covThr);
            bool isHQ = false;
            if (good) {                       // warp-uniform
                // the smallest percentage pc in [0, pct] whose thresholds hold
                // (the reference's loop from pct down to 0 keeps the last one)
                int smallest = 100;
                const int pct = (int)ceilf(fmul_rn(e, 100.0f));
                auto holds = [&](int pc) {
                    const float fac = fdiv_rn((float)pc, 100.0f);
                    const float at = fsub_rn(1.0f, fmul_rn(1.0f, fac));
                    const float mt = fsub_rn(1.0f, fmul_rn(3.0f, fac));
                    return fgeq(avgSup, at) && fgeq(minSup, mt);
                };
                if (pct < 32) {
                    const unsigned bm = __ballot_sync(0xffffffffu, lane <= pct && holds(lane));
                    if (bm) smallest = __ffs(bm) - 1;
                } else {
                    for (int pc = pct; pc >= 0; --pc) if (holds(pc)) smallest = pc;
                }
                isHQ = fgeq((float)minCov, covThr) && fleq((float)smallest, fmul_rn((float)pct, 0.5f));
            }
            if (lane == 0) {
                s_vals[10] = 0;                  // decision positions listed (EMIT)
                s_vals[4] = good;
                s_vals[5] = isHQ;
                s_vals[6] = __float_as_int(avgSup);
                s_vals[7] = __float_as_int(minSup);
                s_vals[8] = minCov;
            }
        }
        __syncthreads();
        allGood = s_vals[4];
        hq = s_vals[5];
    }

    // ---- anchor correction (getCorrectedAnchor, msa.cpp:379-453) ----
    if (V == 0) {
        if (tid == 0) { out.status[ai] = 0; out.nedits[ai] = 0; }
        return;   // nCandidates == 0: not corrected; no candidate corrections either
    }
    int diffs = 0;
    for (int p = tid; p < La; p += BLOCK) {
        const int col = abegin + p;
        const uint32_t ob = s_aelem[p] & 3u;
        uint32_t cb;
        if (allGood) cb = s_cons[col];
        else {
            const int oc = cnt_of(col, ob);   // origCoverages: count of the anchor's base
            cb = (s_support[col] > 0.90f && oc <= 2) ? s_cons[col] : ob;
        }
        aout[p] = "ACGT"[cb];
        diffs += cb != ob;
    }
    int rr[4];
    block_sum4(diffs, 0, 0, 0, rr);
    if (tid == 0) {
        const int nd = rr[0];
        const bool useEdits = !r.ambig[a] && nd <= La / 7;
        out.status[ai] = (uint8_t)(1 | (hq ? 2 : 0) | (useEdits ? 4 : 0));
        out.nedits[ai] = useEdits ? nd : 0;
    }

    // ---- decision columns (correctAnchorClf, corrector.hpp:1448-1472) ----
    // Non-HQ MSAs only: each anchor position whose base differs from the
    // consensus (and whose column reaches clf_min_coverage) becomes a row of
    // 24 features. The plain rule's base stays in aout; with the network
    // deciding, k_clf_apply overwrites it from the row's logit.
    if constexpr (EMIT) {
        if (!hq) {
            // the decision positions are listed first (any order: rows are
            // appended through a global counter), so that their features are
            // computed by consecutive threads instead of by the warps that
            // happen to hold one
            int nm = 0, mxc = 0;
            for (int p = tid; p < La; p += BLOCK) {
                const int col = abegin + p;
                const bool mis = (s_aelem[p] & 3u) != s_cons[col];
                nm += mis;
                mxc = max(mxc, (int)s_cov[col]);
                if (mis && (int)s_cov[col] >= o.clf_min_coverage) s_dec[atomicAdd(&s_vals[10], 1)] = (uint16_t)p;
            }
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                nm += __shfl_xor_sync(0xffffffffu, nm, d);
                mxc = max(mxc, __shfl_xor_sync(0xffffffffu, mxc, d));
            }
            __syncthreads();
            if (lane == 0) { s_red[warp][0] = nm; s_red[warp][1] = mxc; }
            __syncthreads();
            int nmis = 0, maxCov = 0;
#pragma unroll
            for (int w = 0; w < NWARP; ++w) { nmis += s_red[w][0]; maxCov = max(maxCov, s_red[w][1]); }
            const float avgSup = __int_as_float(s_vals[6]), minSup = __int_as_float(s_vals[7]);
            const int minCov = s_vals[8];
            const float E = o.estimated_coverage;
            const int ndec = s_vals[10];
            for (int i = tid; i < ndec; i += BLOCK) {
                const int p = s_dec[i];
                const int col = abegin + p;
                const uint32_t ob = s_aelem[p] & 3u, cb = s_cons[col];
                const float cov = (float)s_cov[col];
                const int oc = cnt_of(col, ob), cc = cnt_of(col, cb);
                const float wsum = s_fw[p], wc = s_fw[mlen + p], wo = s_fw[2 * mlen + p];
                float x[kNumFeatures];
                x[0] = fdiv_rn((float)oc, cov);
                x[1] = fdiv_rn(wo, wsum);
                x[2] = fdiv_rn(wo, (float)oc);
                x[3] = fdiv_rn((float)cc, cov);
                x[4] = s_support[col];
                x[5] = fdiv_rn(wc, (float)cc);
                x[6] = fdiv_rn(wsum, cov);
                x[7] = fdiv_rn(cov, E);
                x[8] = fdiv_rn(wsum, E);
                x[9] = avgSup;
                x[10] = minSup;
                x[11] = fdiv_rn((float)maxCov, E);
                x[12] = fdiv_rn((float)minCov, E);
                x[13] = useQ ? s_qw[s_aelem[p] >> 2] : 1.0f;
                x[14] = fdiv_rn((float)min(p, La - 1 - p), (float)La);
                x[15] = fdiv_rn(fsub_rn(fsub_rn(wsum, wc), wo), wsum);
                const int lo = max(p - 3, 0), hi = min(p + 3, La - 1);
                float ssum = 0.0f, smin = s_support[abegin + lo], qsum = 0.0f;
                for (int q = lo; q <= hi; ++q) {
                    const float sv = s_support[abegin + q];
                    ssum = __fadd_rn(ssum, sv);
                    if (sv < smin) smin = sv;
                    qsum = __fadd_rn(qsum, useQ ? s_qw[s_aelem[q] >> 2] : 1.0f);
                }
                const float nwin = (float)(hi - lo + 1);
                x[16] = fdiv_rn(ssum, nwin);
                x[17] = smin;
                x[18] = fdiv_rn((float)nmis, (float)La);
                int nloc = 0;
                for (int q = max(p - 5, 0); q <= min(p + 5, La - 1); ++q)
                    nloc += q != p && (s_aelem[q] & 3u) != s_cons[abegin + q];
                x[19] = fdiv_rn((float)nloc, 10.0f);
                x[20] = fdiv_rn((float)V, E);
                x[21] = allGood ? 1.0f : 0.0f;
                x[22] = (allGood || (s_support[col] > 0.90f && oc <= 2)) ? 1.0f : 0.0f;
                x[23] = fdiv_rn(qsum, nwin);
                const unsigned long long slot = atomicAdd(out.feat_count, 1ull);
                if (slot >= out.feat_cap) { atomicOr(status, kStatusFeatOverflow); continue; }
                float4* dst = reinterpret_cast<float4*>(out.feat + slot * kNumFeatures);
#pragma unroll
                for (int q = 0; q < kNumFeatures / 4; ++q) dst[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
                out.feat_read[slot] = a;
                out.feat_meta[slot] = (uint32_t)p | (ob << 16) | (cb << 18);
            }
        }
    }

    // ---- candidate correction (getCorrectedCandidates, msa.cpp:457-522) ----
    if (hq && o.correct_candidates) {
        const int ncc = o.new_columns;
        for (int i = tid; i < V; i += BLOCK) {
            uint32_t id; int shift, L; bool fwd;
            if (persistent) {
                const int k = s_alive[i];
                id = s_id[k]; shift = s_beg[k]; L = s_len[k]; fwd = s_fwd[k];
            } else {
                const CandRec rc = recs[off + i];
                id = rc.id; shift = rc.shift; L = rc.len; fwd = rc.orient == 1;
            }
            const int qb = abegin + shift;
            const int qe = qb + L;
            if (!(abegin - ncc <= qb && qb <= abegin + ncc && qe <= aend + ncc)) continue;
            const unsigned long long slot = atomicAdd(out.corr_count, 1ull);
            if (slot >= out.corr_cap) { atomicOr(status, kStatusCorrOverflow); continue; }
            char* dst = out.corr_seq + slot * mlen;
            const uint32_t* row = r.seq + (size_t)id * sp;
            int nd = 0;
            for (int p = 0; p < L; ++p) {
                // forward orientation of the corrected candidate
                const uint32_t cs = fwd ? s_cons[qb + p] : (s_cons[qb + L - 1 - p] ^ 3u);
                dst[p] = "ACGT"[cs];
                nd += cs != base_at(row, p);
            }
            for (int p = L; p < mlen; ++p) dst[p] = 0;   // rows read as zero past the read
            out.corr_id[slot] = id;
            out.corr_anchor[slot] = a;
            out.corr_shift[slot] = shift;
            out.corr_use_edits[slot] = (!r.ambig[id] && nd <= L / 7) ? 1 : 0;
        }
    }
}

// One CTA per anchor, in `order` (e.g. most candidates first) when given;
// the hardware block scheduler hands out the anchors.
template <int BLOCK, int QB, bool EMIT = false>
__global__ void __launch_bounds__(BLOCK, (EMIT ? 768 : 1024) / BLOCK)
k_msa(DevOptions o, DevReads r, uint32_t first, uint32_t count, int jb, const uint32_t* __restrict__ order,
      const uint32_t* __restrict__ cand_ids, const uint32_t* __restrict__ seg_off,
      const uint32_t* __restrict__ seg_cnt, const AlignRes* __restrict__ ares,
      CandRec* __restrict__ recs, MsaOut out, int* __restrict__ status) {
    if (blockIdx.x >= count) return;
    if (*status & kStatusCandOverflow) return;   // batch is repeated with a larger arena
    msa_anchor<BLOCK, QB, EMIT>(o, r, first, order ? order[blockIdx.x] : blockIdx.x, jb, cand_ids, seg_off,
                                seg_cnt, ares, recs, out, status);
}

// Persistent form: a grid of resident CTAs pulls anchors from a device work
// queue (an atomic cursor over `order`) until the batch is done.
template <int BLOCK, int QB, bool EMIT = false>
__global__ void __launch_bounds__(BLOCK, (EMIT ? 768 : 1024) / BLOCK)
k_msa_queue(DevOptions o, DevReads r, uint32_t first, uint32_t count, int jb, const uint32_t* __restrict__ order,
            unsigned int* __restrict__ cursor, const uint32_t* __restrict__ cand_ids,
            const uint32_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_cnt,
            const AlignRes* __restrict__ ares, CandRec* __restrict__ recs, MsaOut out,
            int* __restrict__ status) {
    __shared__ uint32_t s_item;
    if (*status & kStatusCandOverflow) return;
    for (;;) {
        __syncthreads();                      // the previous anchor is done with shared memory
        if (threadIdx.x == 0) s_item = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= count) return;
        msa_anchor<BLOCK, QB, EMIT>(o, r, first, order ? order[it] : it, jb, cand_ids, seg_off, seg_cnt, ares,
                                    recs, out, status);
    }
}

// Longest-processing-time order of a batch's anchors: a counting sort by
// candidate count, most candidates first (order within a count arbitrary:
// anchors are independent, results are written by anchor index).
constexpr int kLptBins = 4096;
static __global__ void k_lpt_hist(const uint32_t* __restrict__ seg_cnt, uint32_t count,
                                  unsigned int* __restrict__ bins) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        atomicAdd(&bins[kLptBins - 1 - min(seg_cnt[i], (uint32_t)(kLptBins - 1))], 1u);
}
// exclusive scan of the bins in place (one CTA of 1024 threads)
static __global__ void k_lpt_scan(unsigned int* __restrict__ bins) {
    __shared__ unsigned int s_part[1024];
    constexpr int per = kLptBins / 1024;
    const int t = threadIdx.x;
    unsigned int loc[per], sum = 0;
#pragma unroll
    for (int k = 0; k < per; ++k) { loc[k] = bins[t * per + k]; sum += loc[k]; }
    s_part[t] = sum;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const unsigned int v = t >= d ? s_part[t - d] : 0u;
        __syncthreads();
        s_part[t] += v;
        __syncthreads();
    }
    unsigned int run = s_part[t] - sum;
#pragma unroll
    for (int k = 0; k < per; ++k) { bins[t * per + k] = run; run += loc[k]; }
}
static __global__ void k_lpt_scatter(const uint32_t* __restrict__ seg_cnt, uint32_t count,
                                     unsigned int* __restrict__ bins, uint32_t* __restrict__ order) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        order[atomicAdd(&bins[kLptBins - 1 - min(seg_cnt[i], (uint32_t)(kLptBins - 1))], 1u)] = i;
}

// Per-alignment order of each anchor's candidate segment by candidate length
// (a counting sort over 16-base length classes, one CTA per anchor): warps of
// k_align then hold pairs of similar scan length. Results stay at their pair
// index, so the MSA still sees candidates in id order.
static __global__ void k_pair_order(const DevReads r, const uint32_t* __restrict__ cand_ids,
                                    const uint32_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_cnt,
                                    uint32_t count, const int* __restrict__ status,
                                    uint32_t* __restrict__ pair_order) {
    constexpr int NB = kMaxLen / 16 + 1;
    __shared__ unsigned int s_bin[NB];
    const uint32_t ai = blockIdx.x;
    if (ai >= count || (*status & kStatusCandOverflow)) return;
    const uint32_t off = seg_off[ai], cnt = seg_cnt[ai];
    for (int b = threadIdx.x; b < NB; b += blockDim.x) s_bin[b] = 0;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) atomicAdd(&s_bin[r.len[cand_ids[off + k]] >> 4], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int run = 0;
        for (int b = 0; b < NB; ++b) { const unsigned int c = s_bin[b]; s_bin[b] = run; run += c; }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x)
        pair_order[off + atomicAdd(&s_bin[r.len[cand_ids[off + k]] >> 4], 1u)] = off + k;
}

// Length classes of the alignment pairs: the plane width (32-base words) the
// longer read of a pair needs, 4 / 5 / 6 / 8, so that each class runs the
// k_align instance of its width (fewer registers for short pairs, lanes of
// similar lengths). cls[c] = {offset in the class list, pairs}; within a
// class, warps keep the pair order they read (warp-aggregated cursors).
constexpr int kAlignClasses = 4;
__host__ __device__ inline int align_class_width(int c) { return c == 0 ? 4 : c == 1 ? 5 : c == 2 ? 6 : 8; }
__device__ __forceinline__ int align_class_of(int L) {
    const int nw = (L + 31) >> 5;
    return nw <= 4 ? 0 : nw == 5 ? 1 : nw == 6 ? 2 : 3;
}
__device__ __forceinline__ int pair_class(const DevReads& r, uint32_t first, const uint32_t* cand_ids,
                                          const uint32_t* cand_anchor, unsigned long long i) {
    return align_class_of(max(r.len[first + cand_anchor[i]], r.len[cand_ids[i]]));
}
static __global__ void k_pair_class_count(DevReads r, uint32_t first, const uint32_t* __restrict__ cand_ids,
                                          const uint32_t* __restrict__ cand_anchor,
                                          const unsigned long long* __restrict__ total_ptr, unsigned long long cap,
                                          const int* __restrict__ status, const uint32_t* __restrict__ pair_order,
                                          uint2* __restrict__ cls) {
    if (*status & kStatusCandOverflow) return;
    const unsigned long long total = *total_ptr;
    if (total > cap) return;
    const int lane = threadIdx.x & 31;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long s0 = (unsigned long long)blockIdx.x * blockDim.x; s0 < total; s0 += stride) {
        const unsigned long long slot = s0 + threadIdx.x;
        const bool act = slot < total;
        const int c = act ? pair_class(r, first, cand_ids, cand_anchor, pair_order ? pair_order[slot] : slot) : -1;
#pragma unroll
        for (int k = 0; k < kAlignClasses; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, c == k);
            if (m && lane == 0) atomicAdd(&cls[k].y, (unsigned)__popc(m));
        }
    }
}
static __global__ void k_pair_class_offsets(uint2* __restrict__ cls, unsigned int* __restrict__ cursor) {
    if (threadIdx.x != 0) return;
    unsigned run = 0;
    for (int k = 0; k < kAlignClasses; ++k) { cls[k].x = run; cursor[k] = run; run += cls[k].y; }
}
static __global__ void k_pair_class_scatter(DevReads r, uint32_t first, const uint32_t* __restrict__ cand_ids,
                                            const uint32_t* __restrict__ cand_anchor,
                                            const unsigned long long* __restrict__ total_ptr, unsigned long long cap,
                                            const int* __restrict__ status, const uint32_t* __restrict__ pair_order,
                                            unsigned int* __restrict__ cursor, uint32_t* __restrict__ list) {
    if (*status & kStatusCandOverflow) return;
    const unsigned long long total = *total_ptr;
    if (total > cap) return;
    const int lane = threadIdx.x & 31;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long s0 = (unsigned long long)blockIdx.x * blockDim.x; s0 < total; s0 += stride) {
        const unsigned long long slot = s0 + threadIdx.x;
        const bool act = slot < total;
        const uint32_t i = act ? (pair_order ? pair_order[slot] : (uint32_t)slot) : 0u;
        const int c = act ? pair_class(r, first, cand_ids, cand_anchor, i) : -1;
#pragma unroll
        for (int k = 0; k < kAlignClasses; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, c == k);
            if (!m) continue;
            unsigned b = 0;
            if (lane == 0) b = atomicAdd(&cursor[k], (unsigned)__popc(m));
            b = __shfl_sync(0xffffffffu, b, 0);
            if (c == k) list[b + __popc(m & ((1u << lane) - 1u))] = i;
        }
    }
}

// The network's verdict on each decision column of the batch: the consensus
// base where the logit is positive, else the original base.
static __global__ void k_clf_apply(const uint32_t* __restrict__ feat_read, const uint32_t* __restrict__ feat_meta,
                            const float* __restrict__ logit, const unsigned long long* __restrict__ count,
                            unsigned long long cap, uint32_t first, int mlen, char* __restrict__ seq,
                            uint8_t* __restrict__ touched) {
    const unsigned long long n = min(*count, cap);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t meta = feat_meta[i];
        const uint32_t ai = feat_read[i] - first;
        const uint32_t b = logit[i] > 0.0f ? (meta >> 18) & 3u : (meta >> 16) & 3u;
        seq[(size_t)ai * mlen + (meta & 0xFFFFu)] = "ACGT"[b];
        touched[ai] = 1;
    }
}

// Edit counts of the anchors whose corrected sequence k_clf_apply changed
// (makeOutputOfTask, corrector.hpp:1648-1675): one warp per anchor.
static __global__ void k_clf_recount(DevReads r, uint32_t first, uint32_t count, const uint8_t* __restrict__ touched,
                              const char* __restrict__ seq, uint8_t* __restrict__ status,
                              int32_t* __restrict__ nedits) {
    const int lane = threadIdx.x & 31;
    const uint32_t ai = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (ai >= count || !touched[ai]) return;
    const uint32_t a = first + ai;
    const int La = r.len[a];
    const uint32_t* row = r.seq + (size_t)a * r.seq_pitch;
    const char* s = seq + (size_t)ai * r.max_len;
    int nd = 0;
    for (int p = lane; p < La; p += 32) nd += "ACGT"[base_at(row, p)] != s[p];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) nd += __shfl_xor_sync(0xffffffffu, nd, d);
    if (lane == 0) {
        const bool useEdits = !r.ambig[a] && nd <= La / 7;
        status[ai] = (uint8_t)((status[ai] & ~4u) | (useEdits ? 4u : 0u));
        nedits[ai] = useEdits ? nd : 0;
    }
}

// Signatures of all reads (for table construction): one warp per read.
static __global__ void k_signatures(DevOptions o, DevReads r, uint32_t first, uint32_t count,
                             unsigned long long* __restrict__ sig) {
    const int lane = threadIdx.x & 31;
    const uint32_t ri = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (ri >= count) return;
    const uint32_t id = first + ri;
    const int L = r.len[id];
    const int h = o.num_maps;
    const uint32_t* row = r.seq + (size_t)id * r.seq_pitch;
    unsigned long long mine[2] = {~0ull, ~0ull};  // maps lane and lane+32
    unsigned long long alt[2] = {~0ull, ~0ull};
    if (L >= o.k) {
        const int npos = L - o.k + 1;
        const int rcshift = 64 - 2 * o.k;
        for (int p0 = 0; p0 < npos; p0 += 32) {
            // each lane builds one canonical k-mer, then all lanes hash all 32
            unsigned long long cn = 0;
            const int p = p0 + lane;
            if (p < npos) {
                const int w = p >> 4, of = p & 15;
                const uint32_t s0 = __ldg(row + w);
                const uint32_t s1 = (w + 1 < r.seq_pitch) ? __ldg(row + w + 1) : 0u;
                const uint32_t s2 = (w + 2 < r.seq_pitch) ? __ldg(row + w + 2) : 0u;
                const unsigned long long hi = ((unsigned long long)s0 << 32) | s1;
                const unsigned long long top = of ? (hi << (2 * of)) | ((unsigned long long)s2 >> (32 - 2 * of)) : hi;
                const unsigned long long fw = top >> (64 - 2 * o.k);
                const unsigned long long rv = revcomp64(fw) >> rcshift;
                cn = fw < rv ? fw : rv;
            }
            // two k-mers per step into separate minima (the min chains of a
            // lane overlap; an odd count hashes the last k-mer twice)
            const int nv = min(32, npos - p0);
            for (int q = 0; q < nv; q += 2) {
                const unsigned long long k0 = __shfl_sync(0xffffffffu, cn, q);
                const unsigned long long k1 = __shfl_sync(0xffffffffu, cn, q + 1 < nv ? q + 1 : q);
                if (lane < h) {
                    const unsigned long long v0 = murmur64(k0 + lane), v1 = murmur64(k1 + lane);
                    mine[0] = v0 < mine[0] ? v0 : mine[0];
                    alt[0] = v1 < alt[0] ? v1 : alt[0];
                }
                if (lane + 32 < h) {
                    const unsigned long long v0 = murmur64(k0 + lane + 32), v1 = murmur64(k1 + lane + 32);
                    mine[1] = v0 < mine[1] ? v0 : mine[1];
                    alt[1] = v1 < alt[1] ? v1 : alt[1];
                }
            }
        }
    }
    mine[0] = alt[0] < mine[0] ? alt[0] : mine[0];
    mine[1] = alt[1] < mine[1] ? alt[1] : mine[1];
    if (lane < h) sig[(size_t)ri * h + lane] = mine[0] & o.kmer_mask;
    if (lane + 32 < h) sig[(size_t)ri * h + lane + 32] = mine[1] & o.kmer_mask;
}

}  // namespace careb200
