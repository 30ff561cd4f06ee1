// noalloc.cu -- correction of a batch of anchors without any allocation.
//
// Some callers cannot call cudaMalloc: code that runs on memory a host
// framework has already laid out (a fixed device pool, buffers mapped from
// another process) or that must not change the device's memory map once it
// is running. For them care_b200_correct_range_noalloc() takes every input
// and output as a device pointer the caller owns and keeps all of its
// working memory (candidate lists, alignments, filtered candidates, counters)
// in one file-scope device array of fixed size, kNoAllocScratchBytes.
#include "../../include/care_b200.h"
#include "hostio.hpp"
#include "kernels.cuh"

#include <algorithm>
#include <mutex>

using namespace careb200;

namespace {

constexpr uint32_t kNoAllocMaxAnchors = CARE_B200_NOALLOC_MAX_ANCHORS;
constexpr unsigned long long kNoAllocMaxPairs = CARE_B200_NOALLOC_MAX_PAIRS;

// Byte offsets of the parts of the scratch array (each 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffCounters = 0;                                          // u64[8]
constexpr size_t kOffStatus = 64;                                           // int[4]
constexpr size_t kOffSegOff = 256;
constexpr size_t kOffSegCnt = align256(kOffSegOff + 4ull * kNoAllocMaxAnchors);
constexpr size_t kOffCandIds = align256(kOffSegCnt + 4ull * kNoAllocMaxAnchors);
constexpr size_t kOffCandAnchor = align256(kOffCandIds + 4ull * kNoAllocMaxPairs);
constexpr size_t kOffAres = align256(kOffCandAnchor + 4ull * kNoAllocMaxPairs);
constexpr size_t kOffRecs = align256(kOffAres + sizeof(AlignRes) * kNoAllocMaxPairs);
constexpr size_t kNoAllocScratchBytes = align256(kOffRecs + sizeof(CandRec) * kNoAllocMaxPairs);
static_assert(kNoAllocScratchBytes < (48ull << 20), "scratch must stay modest");

// The scratch. Every device that loads the library holds this array until the
// process exits. In host code its name is only a host-side stand-in: kernels
// get the device address fetched with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Once per device, with that device current: the scratch address and the
// quality weight table of this module.
int setup_device(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev]) {
        *out = g_scratch_ptr[dev];
        return CARE_B200_OK;
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CARE_B200_ECUDA;
    float qw[256];
    quality_weights(qw);
    if (cudaMemcpyToSymbol(c_qweight, qw, sizeof(qw)) != cudaSuccess) return CARE_B200_ECUDA;
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    *out = g_scratch_ptr[dev];
    return CARE_B200_OK;
}

constexpr int kStatusBadLength = 1 << 16;    // a read length outside [0, max_length]

// Every read length within [0, max_len]: the kernels size their shared memory
// and registers from max_len and index by the lengths.
__global__ void k_check_lengths(const int* __restrict__ len, uint32_t n, int max_len, int* __restrict__ status) {
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int L = len[i];
        bad |= L < 0 || L > max_len;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatusBadLength);
}

}  // namespace

extern "C" int care_b200_correct_range_noalloc(const care_b200_options* opt, const care_b200_device_reads* reads,
                                               const care_b200_device_tables* tables, uint32_t first_anchor,
                                               uint32_t num_anchors, uint8_t* status, int32_t* num_edits,
                                               char* sequences, void* stream) {
    if (!opt || !reads || !tables || !status || !num_edits || !sequences) return CARE_B200_EINVAL;
    if (num_anchors == 0) return CARE_B200_OK;
    if (opt->correct_candidates) return CARE_B200_EINVAL;                 // anchor correction only
    if (opt->correction_type != 0) return CARE_B200_EINVAL;               // plain rule only
    if (opt->num_maps < 1 || opt->num_maps > kMaxMaps || tables->num_maps != opt->num_maps) return CARE_B200_EINVAL;
    if (opt->kmerlength < 1 || opt->kmerlength > 32) return CARE_B200_EINVAL;
    if (opt->quality_bits != 1 && opt->quality_bits != 2 && opt->quality_bits != 8) return CARE_B200_EINVAL;
    if (!reads->packed || !reads->lengths || !reads->ambiguous || reads->num_reads == 0) return CARE_B200_EINVAL;
    if (opt->use_quality && !reads->quals) return CARE_B200_EINVAL;
    if (!tables->descs || !tables->slots || !tables->values) return CARE_B200_EINVAL;
    if ((uint64_t)first_anchor + num_anchors > reads->num_reads) return CARE_B200_EINVAL;
    if (opt->paired_end && ((first_anchor | num_anchors) & 1)) return CARE_B200_EINVAL;
    if (num_anchors > kNoAllocMaxAnchors) return CARE_B200_ELIMIT;
    if (reads->max_length < 1 || reads->max_length > kMaxLen) return CARE_B200_ELIMIT;
    if ((size_t)(reads->max_length + 15) / 16 > reads->pitch_ints) return CARE_B200_EINVAL;
    if (reads->pitch_ints > (size_t)kMaxLen / 16) return CARE_B200_EINVAL;
    if (opt->use_quality &&
        ((size_t)((int64_t)reads->max_length * opt->quality_bits + 31) / 32 > reads->qual_pitch_ints ||
         reads->qual_pitch_ints > (size_t)kMaxLen * opt->quality_bits / 32))
        return CARE_B200_EINVAL;
    if (tables->threshold < 0 || tables->threshold > 65535) return CARE_B200_EINVAL;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CARE_B200_ECUDA;
    unsigned char* scratch = nullptr;
    const int rc = setup_device(dev, &scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    DevOptions o{};
    o.k = opt->kmerlength;
    o.num_maps = opt->num_maps;
    o.min_overlap = opt->min_overlap;
    o.new_columns = opt->new_columns_to_correct;
    o.use_quality = opt->use_quality && reads->quals != nullptr;
    o.quality_bits = opt->quality_bits;
    o.exclude_ambiguous = opt->exclude_ambiguous;
    o.correct_candidates = 0;
    o.paired_end = opt->paired_end;
    if (tables->threshold > 0) {
        o.threshold = tables->threshold;                                 // the tables' own (e.g. from a file)
    } else {
        const int cov = (int)opt->estimated_coverage;
        int t = (int)(cov * 2.5f);
        t = t > 65535 ? 65535 : t;
        o.threshold = t < 10 ? 10 : t;                                   // minhasherlimit.hpp:9-15
    }
    o.coverage_int = (int)opt->estimated_coverage;
    o.correction_type = opt->correction_type;
    o.max_error_rate = opt->max_error_rate;
    o.min_overlap_ratio = opt->min_overlap_ratio;
    o.estimated_errorrate = opt->estimated_errorrate;
    o.estimated_coverage = opt->estimated_coverage;
    o.m_coverage = opt->m_coverage;
    o.paired_filter_threshold = opt->paired_filter_threshold;
    o.kmer_mask = ~0ull >> ((32 - opt->kmerlength) * 2);

    DevReads r{};
    r.seq = reads->packed;
    r.qual = o.use_quality ? reads->quals : nullptr;
    r.len = reads->lengths;
    r.ambig = reads->ambiguous;
    r.seq_pitch = (int)reads->pitch_ints;
    r.qual_pitch = o.use_quality ? (int)reads->qual_pitch_ints : 0;
    r.max_len = reads->max_length;
    r.n = reads->num_reads;

    unsigned long long* counters = reinterpret_cast<unsigned long long*>(scratch + kOffCounters);
    int* dstatus = reinterpret_cast<int*>(scratch + kOffStatus);
    uint32_t* seg_off = reinterpret_cast<uint32_t*>(scratch + kOffSegOff);
    uint32_t* seg_cnt = reinterpret_cast<uint32_t*>(scratch + kOffSegCnt);
    uint32_t* cand_ids = reinterpret_cast<uint32_t*>(scratch + kOffCandIds);
    uint32_t* cand_anchor = reinterpret_cast<uint32_t*>(scratch + kOffCandAnchor);
    AlignRes* ares = reinterpret_cast<AlignRes*>(scratch + kOffAres);
    CandRec* recs = reinterpret_cast<CandRec*>(scratch + kOffRecs);

    // the counters and status word keep the previous call's values: clear them
    if (cudaMemsetAsync(scratch, 0, 256, st) != cudaSuccess) return CARE_B200_ECUDA;
    if (cudaMemsetAsync(sequences, 0, (size_t)num_anchors * reads->max_length, st) != cudaSuccess) return CARE_B200_ECUDA;
    // lengths beyond max_length would take the kernels past their buffers:
    // rejected before any of them runs
    {
        const unsigned cb = (unsigned)std::min<uint64_t>((r.n + 255) / 256, 1024);
        k_check_lengths<<<cb, 256, 0, st>>>(r.len, r.n, r.max_len, dstatus);
        int hs = 0;
        if (cudaMemcpyAsync(&hs, dstatus, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CARE_B200_ECUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return CARE_B200_ECUDA;
        if (hs & kStatusBadLength) return CARE_B200_EINVAL;
    }

    const int h = o.num_maps;
    const size_t tmax = (size_t)h * o.threshold;
    int set_log2 = 6;                 // at least 64 entries: the set and the sort pad to 64 and 32
    while ((size_t)1 << set_log2 < (tmax * 4 + 2) / 3 + 1) set_log2++;
    const size_t cand_smem = CandSmem::total(r.max_len, 128 / h, h, r.seq_pitch, 1 << set_log2);
    if (cand_smem > 227 * 1024) return CARE_B200_ELIMIT;
    if (cudaFuncSetAttribute(k_candidates<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cand_smem) != cudaSuccess)
        return CARE_B200_ECUDA;
    k_candidates<128><<<num_anchors, 128, cand_smem, st>>>(
        o, r, static_cast<const TableDesc*>(tables->descs), static_cast<const Slot*>(tables->slots), tables->values,
        nullptr, first_anchor, num_anchors, set_log2, nullptr, nullptr, cand_ids, cand_anchor, seg_off, seg_cnt, counters, kNoAllocMaxPairs,
        dstatus);
    // the pairs the candidate pass found size the alignment grid; a count
    // above the array's pair capacity ends the call here
    unsigned long long npairs = 0;
    if (cudaMemcpyAsync(&npairs, counters, sizeof(npairs), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return CARE_B200_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CARE_B200_ECUDA;
    if (npairs > kNoAllocMaxPairs) return CARE_B200_ELIMIT;
    const unsigned ablocks = (unsigned)std::max<unsigned long long>((npairs + 127) / 128, 1);
    const int nw = (r.max_len + 31) / 32;
#define LAUNCH_ALIGN(NW)                                                                                    \
    k_align<128, NW><<<ablocks, 128, 0, st>>>(o, r, first_anchor, cand_ids, cand_anchor, seg_off, seg_cnt,  \
                                              counters, kNoAllocMaxPairs, dstatus, ares, nullptr, nullptr, nullptr, nullptr, nullptr)
    if (nw <= 4) LAUNCH_ALIGN(4);
    else if (nw <= 5) LAUNCH_ALIGN(5);
    else if (nw <= 6) LAUNCH_ALIGN(6);
    else LAUNCH_ALIGN(8);
#undef LAUNCH_ALIGN
    MsaOut mo{};
    mo.status = status;
    mo.nedits = num_edits;
    mo.seq = sequences;
    mo.corr_count = counters + 1;
    mo.corr_cap = 0;                     // no candidate corrections in this entry point
    // widest possible MSA: La + 2*Lmax - 2*minoverlap(La), maximised over La
    int maxcols = 1;
    for (int la = 1; la <= r.max_len; ++la) {
        const int lo = (int)((float)la * opt->min_overlap_ratio);
        const int mo2 = lo > opt->min_overlap ? lo : opt->min_overlap;
        const int c = la + 2 * r.max_len - 2 * (mo2 < r.max_len ? mo2 : r.max_len);
        maxcols = c > maxcols ? c : maxcols;
    }
    const int jb = (maxcols + 127) / 128;
    const int qb = !o.use_quality ? 0 : o.quality_bits == 1 ? 1 : o.quality_bits == 2 ? 2 : 8;
    const size_t msmem = msa_smem_bytes(r.max_len, r.seq_pitch, r.qual_pitch, qb, false, 128 * jb);
#define LAUNCH_MSA(QB)                                                                                   \
    do {                                                                                                  \
        if (cudaFuncSetAttribute(k_msa<128, QB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem) \
            != cudaSuccess)                                                                               \
            return CARE_B200_ECUDA;                                                                       \
        k_msa<128, QB><<<num_anchors, 128, msmem, st>>>(o, r, first_anchor, num_anchors, jb, nullptr,     \
                                                        cand_ids, seg_off, seg_cnt, ares, recs, mo,       \
                                                        dstatus);                                         \
    } while (0)
    if (!o.use_quality) LAUNCH_MSA(0);
    else if (o.quality_bits == 1) LAUNCH_MSA(1);
    else if (o.quality_bits == 2) LAUNCH_MSA(2);
    else LAUNCH_MSA(8);
#undef LAUNCH_MSA
    if (cudaGetLastError() != cudaSuccess) return CARE_B200_ECUDA;
    int hstatus = 0;
    if (cudaMemcpyAsync(&hstatus, dstatus, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CARE_B200_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CARE_B200_ECUDA;
    if (hstatus & (kStatusCandOverflow | kStatusColumns)) return CARE_B200_ELIMIT;
    return CARE_B200_OK;
}
