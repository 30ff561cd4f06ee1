// capi.cu -- the C ABI (include/care_b200.h): context, device-resident read
// storage and minhash tables, the batched correction pipeline, results.
#include "../../include/care_b200.h"
#include "hostio.hpp"
#include "readfile.hpp"
#include "kernels.cuh"
#include "mlp.hpp"
#include "parse.hpp"
#include "tables.hpp"

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

using namespace careb200;

namespace {

// Device allocation that frees itself.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        const cudaError_t e = cudaMalloc(&p, n ? n : 16);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void adopt(void* q, size_t n) { release(); p = q; bytes = n; }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Pinned host allocation that frees itself.
struct HBuf {
    void* p = nullptr;
    size_t bytes = 0;
    HBuf() = default;
    HBuf(const HBuf&) = delete;
    HBuf& operator=(const HBuf&) = delete;
    ~HBuf() { release(); }
    void release() { if (p) cudaFreeHost(p); p = nullptr; bytes = 0; }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        const cudaError_t e = cudaMallocHost(&p, n ? n : 16);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Host threads that copy one buffer in equal parts, kept for the context's
// life: a copy of pageable caller memory into pinned staging runs at one
// core's copy rate per thread, and starting threads per 16 MB chunk costs
// as much as the copy.
class CopyPool {
public:
    explicit CopyPool(unsigned n) : n_(std::max(1u, n)) {
        for (unsigned i = 1; i < n_; ++i) th_.emplace_back([this, i] { run(i); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            quit_ = true;
        }
        go_.notify_all();
        for (auto& t : th_) t.join();
    }
    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;
    // copies len bytes from src to dst; the calling thread takes part 0
    void copy(void* dst, const void* src, size_t len) {
        {
            std::lock_guard<std::mutex> g(m_);
            dst_ = static_cast<char*>(dst);
            src_ = static_cast<const char*>(src);
            len_ = len;
            part_ = (len + n_ - 1) / n_;
            pending_ = n_ - 1;
            ++gen_;
        }
        go_.notify_all();
        part(0);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }

private:
    void part(unsigned i) {
        const size_t a = (size_t)i * part_;
        if (a < len_) std::memcpy(dst_ + a, src_ + a, std::min(part_, len_ - a));
    }
    void run(unsigned i) {
        unsigned long long seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            go_.wait(lk, [&] { return quit_ || gen_ != seen; });
            if (quit_) return;
            seen = gen_;
            lk.unlock();
            part(i);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    unsigned n_;
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable go_, done_;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t len_ = 0, part_ = 0;
    unsigned pending_ = 0;
    unsigned long long gen_ = 0;
    bool quit_ = false;
};

constexpr int kCandBlock = 128;
constexpr int kAlignBlock = 128;
constexpr int kMsaBlock = 128;

}  // namespace

// The launch mapping of a new context: one kernel per stage in anchor order,
// 4 MSA warps, 128-thread alignment CTAs, a 1024-entry candidate set.
constexpr care_b200_tuning kDefaultTuning{0, 0, 4, 128, 0, 0, 0, 10, 0, 0};

// Largest candidate arena of one batch: pair indices and offsets are 32-bit.
constexpr unsigned long long kMaxBatchPairs = 0xffffffffull;

struct care_b200_ctx {
    care_b200_options opt{};
    std::string err;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // around each launch of the last signature pass (pairs; the pass may be
    // split into chunks interleaved with the upload of the reads)
    std::vector<cudaEvent_t> sig_ev;
    int sig_used = 0;
    float last_ms = 0.f, stage_ms[4] = {0.f, 0.f, 0.f, 0.f};

    // read storage
    uint32_t n = 0;
    int max_len = 0, seq_pitch = 0, qual_pitch = 0;
    bool has_qual = false;
    DBuf d_seq, d_qual, d_len, d_ambig;
    std::vector<uint8_t> h_ambig;
    std::vector<int32_t> h_len;
    HostReads reads;                  // set when loaded from files
    bool have_records = false;

    // tables
    int num_maps = 0, threshold = 0;
    DBuf d_slots, d_values, d_tdesc;
    std::vector<std::vector<uint64_t>> t_keys;
    std::vector<std::vector<uint32_t>> t_off, t_val;
    bool tables_ready = false;
    uint32_t tables_reads = 0;        // storage size the tables were built for
    // minhash signatures of all reads (n * num_maps keys), resident so the
    // candidate stage only looks them up
    DBuf d_sigs;
    int sigs_maps = 0;                // 0: not computed for the current storage

    // batch scratch
    DBuf d_seg_off, d_seg_cnt, d_cand_ids, d_cand_anchor, d_ares, d_recs, d_counters, d_status;
    unsigned long long cand_cap = 0;
    DBuf d_st, d_ned, d_oseq;
    DBuf d_cid, d_canc, d_cshift, d_cue, d_cseq;
    unsigned long long corr_cap = 0;
    HBuf h_small;
    HBuf h_text;                      // input files' bytes (records parsed on the device point into it)
    // host -> device staging of uploads: two pinned chunks per copy stream
    HBuf h_stage[2][2];
    std::unique_ptr<CopyPool> copy_pool;          // host threads filling the staging chunks
    cudaEvent_t stage_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cudaStream_t copy_stream = nullptr;
    cudaStream_t copy_stream2 = nullptr;          // quality words while the sequences upload

    // learned decision: parameters, decision-column rows of a batch
    DBuf d_mlp, d_mlp_err;
    bool mlp_set = false;
    bool collect = false;             // keep the rows of the current call
    DBuf d_fx, d_fread, d_fmeta, d_flogit, d_touched;
    unsigned long long feat_cap = 0;
    std::vector<float> r_fx, r_flogit;
    std::vector<uint32_t> r_fread, r_fmeta;

    // launch mapping (care_b200_set_tuning) and its scratch
    care_b200_tuning tune = kDefaultTuning;
    DBuf d_order, d_bins, d_pair_order, d_pair_work, d_spill, d_pair_class, d_cls;
    cudaGraphExec_t gexec = nullptr;
    int sms = 0;

    // results of the last call (pinned host)
    HBuf r_status, r_nedits, r_seq;
    HBuf r_cid, r_canc, r_cshift, r_cue, r_cseq;
    uint64_t r_ncand = 0, r_pairs = 0, r_words = 0, r_elems = 0, r_batches = 0, r_launches = 0, r_spilled = 0;
    uint64_t r_rb_elems = 0, r_rb_anchors = 0;
    uint64_t r_run_words = 0;
    bool count_words = false;         // the alignment's statistics form (care_b200_count_word_compares)
    double pairs_per_anchor = 96.0;   // seen in the last correction call (automatic batch size)
    uint32_t r_first = 0, r_count = 0;
    bool r_valid = false;
};

namespace {

int fail(care_b200_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(care_b200_ctx* c, cudaError_t e, const char* where) {
    return fail(c, CARE_B200_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call, where)                                             \
    do {                                                            \
        const cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where);    \
    } while (0)

DevOptions make_dev_options(const care_b200_ctx* ctx) {
    const care_b200_options& o = ctx->opt;
    DevOptions d{};
    d.k = o.kmerlength;
    d.num_maps = ctx->num_maps ? ctx->num_maps : o.num_maps;
    d.min_overlap = o.min_overlap;
    d.new_columns = o.new_columns_to_correct;
    d.use_quality = o.use_quality && ctx->has_qual;
    d.quality_bits = o.quality_bits;
    d.exclude_ambiguous = o.exclude_ambiguous;
    d.correct_candidates = o.correct_candidates;
    d.paired_end = o.paired_end;
    d.threshold = ctx->threshold;
    d.coverage_int = (int)o.estimated_coverage;
    d.correction_type = o.correction_type;
    d.clf_mode = o.correction_type == 1 ? 2 : (ctx->collect ? 1 : 0);
    d.clf_min_coverage = o.clf_min_coverage;
    d.max_error_rate = o.max_error_rate;
    d.min_overlap_ratio = o.min_overlap_ratio;
    d.estimated_errorrate = o.estimated_errorrate;
    d.estimated_coverage = o.estimated_coverage;
    d.m_coverage = o.m_coverage;
    d.paired_filter_threshold = o.paired_filter_threshold;
    d.kmer_mask = ~0ull >> ((32 - o.kmerlength) * 2);
    return d;
}

DevReads make_dev_reads(const care_b200_ctx* ctx) {
    DevReads r{};
    r.seq = ctx->d_seq.as<uint32_t>();
    r.qual = ctx->has_qual ? ctx->d_qual.as<uint32_t>() : nullptr;
    r.len = ctx->d_len.as<int32_t>();
    r.ambig = ctx->d_ambig.as<uint8_t>();
    r.seq_pitch = ctx->seq_pitch;
    r.qual_pitch = ctx->qual_pitch;
    r.max_len = ctx->max_len;
    r.n = ctx->n;
    return r;
}

// calculateResultsPerMapThreshold (minhasherlimit.hpp:9-15) of int(coverage)
int results_per_map_threshold(float coverage) {
    const int cov = (int)coverage;
    int r = (int)(cov * 2.5f);
    r = std::min(r, 65535);
    return std::max(10, r);
}

uint64_t host_murmur64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// minhash signatures of reads [b, e) for `maps` hash functions into d_sigs
// (allocated for every read by the caller), each launch timed by an event pair
int signatures_range(care_b200_ctx* ctx, int maps, uint32_t b, uint32_t e) {
    DevOptions o = make_dev_options(ctx);
    o.num_maps = maps;
    const DevReads r = make_dev_reads(ctx);
    const uint32_t chunk = 1u << 20;
    for (; b < e; b += chunk) {
        const uint32_t cnt = std::min(chunk, e - b);
        if ((size_t)ctx->sig_used + 2 > ctx->sig_ev.size()) {
            cudaEvent_t a2[2];
            for (auto& x : a2) CK(cudaEventCreate(&x), "cudaEventCreate");
            ctx->sig_ev.push_back(a2[0]);
            ctx->sig_ev.push_back(a2[1]);
        }
        const int wpb = 8;
        CK(cudaEventRecord(ctx->sig_ev[ctx->sig_used], ctx->stream), "event");
        k_signatures<<<(cnt + wpb - 1) / wpb, 32 * wpb, 0, ctx->stream>>>(
            o, r, b, cnt, ctx->d_sigs.as<unsigned long long>() + (size_t)b * maps);
        CK(cudaGetLastError(), "k_signatures");
        CK(cudaEventRecord(ctx->sig_ev[ctx->sig_used + 1], ctx->stream), "event");
        ctx->sig_used += 2;
    }
    return CARE_B200_OK;
}

// minhash signatures of every read for `maps` hash functions into d_sigs
int compute_signatures(care_b200_ctx* ctx, int maps) {
    CK(ctx->d_sigs.ensure((size_t)ctx->n * maps * 8), "alloc signatures");
    ctx->sig_used = 0;
    if (int rc = signatures_range(ctx, maps, 0, ctx->n)) return rc;
    ctx->sigs_maps = maps;
    return CARE_B200_OK;
}

// Host -> device copy of pageable caller memory through two pinned chunks of
// staging slot `slot`: host threads fill one chunk while the copy engine
// drains the other. Asynchronous on `st` (the caller synchronises).
// on_chunk(end, done): called after the copy of bytes [.., end) is enqueued
// on st; the event `done` completes with that copy.
int staged_upload(care_b200_ctx* ctx, int slot, void* dst, const void* src, size_t bytes, cudaStream_t st,
                  const std::function<int(size_t, cudaEvent_t)>& on_chunk = nullptr) {
    constexpr size_t kChunk = 16u << 20;
    if (bytes <= kChunk / 4) {               // small: one pinned copy is not worth it
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "upload");
        CK(cudaStreamSynchronize(st), "upload");
        if (on_chunk) if (int rc = on_chunk(bytes, nullptr)) return rc;
        return CARE_B200_OK;
    }
    for (auto& b : ctx->h_stage[slot]) CK(b.ensure(kChunk), "alloc staging");
    if (!ctx->copy_pool) ctx->copy_pool.reset(new CopyPool(std::min(16u, std::thread::hardware_concurrency())));
    size_t off = 0;
    for (int i = 0; off < bytes; ++i, off += kChunk) {
        const int b = i & 1;
        const size_t len = std::min(kChunk, bytes - off);
        CK(cudaEventSynchronize(ctx->stage_ev[slot][b]), "staging");   // the chunk's previous copy is done
        char* pin = ctx->h_stage[slot][b].as<char>();
        ctx->copy_pool->copy(pin, static_cast<const char*>(src) + off, len);
        CK(cudaMemcpyAsync(static_cast<char*>(dst) + off, pin, len, cudaMemcpyHostToDevice, st), "upload");
        CK(cudaEventRecord(ctx->stage_ev[slot][b], st), "staging");
        if (on_chunk) if (int rc = on_chunk(off + len, ctx->stage_ev[slot][b])) return rc;
    }
    return CARE_B200_OK;
}

int validate_options(care_b200_ctx* ctx, const care_b200_options& o) {
    // ProgramOptions::isValid, src/options.cpp:387-480, plus this library's limits
    if (o.max_error_rate < 0.f || o.max_error_rate > 1.f) return fail(ctx, CARE_B200_EINVAL, "maxmismatchratio must be in [0,1]");
    if (o.min_overlap < 1) return fail(ctx, CARE_B200_EINVAL, "min_overlap must be > 0");
    if (o.min_overlap_ratio < 0.f || o.min_overlap_ratio > 1.f) return fail(ctx, CARE_B200_EINVAL, "min_overlap_ratio must be in [0,1]");
    if (!(o.estimated_coverage > 0.f)) return fail(ctx, CARE_B200_EINVAL, "estimatedCoverage must be > 0");
    if (!(o.estimated_errorrate > 0.f)) return fail(ctx, CARE_B200_EINVAL, "estimatedErrorrate must be > 0");
    if (o.num_maps < 1 || o.num_maps > kMaxMaps) return fail(ctx, CARE_B200_EINVAL, "number of hash maps must be in [1,48]");
    if (o.kmerlength < 1 || o.kmerlength > 32) return fail(ctx, CARE_B200_EINVAL, "kmer length must be in [1,32]");
    if (o.quality_bits != 1 && o.quality_bits != 2 && o.quality_bits != 8) return fail(ctx, CARE_B200_EINVAL, "qualityScoreBits must be 1, 2 or 8");
    if (o.correction_type != 0 && o.correction_type != 1) return fail(ctx, CARE_B200_EINVAL, "correction_type must be 0 or 1");
    if (o.clf_min_coverage < 0) return fail(ctx, CARE_B200_EINVAL, "clf_min_coverage must be >= 0");
    return CARE_B200_OK;
}

}  // namespace

extern "C" {

void care_b200_default_options(care_b200_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->kmerlength = 20;
    o->num_maps = 48;
    o->min_overlap = 30;
    o->max_error_rate = 0.2f;
    o->min_overlap_ratio = 0.30f;
    o->estimated_errorrate = 0.06f;
    o->estimated_coverage = 1.0f;
    o->m_coverage = 0.6f;
    o->paired_filter_threshold = 0.06f;
    o->new_columns_to_correct = 15;
    o->quality_bits = 8;
    o->threads = 0;
    o->device = 0;
    o->clf_min_coverage = 3;
}

static int care_b200_create_impl(const care_b200_options* opt, care_b200_ctx** out);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_create(const care_b200_options* opt, care_b200_ctx** out) {
    try {
        return care_b200_create_impl(opt, out);
    } catch (const std::exception&) {
        return CARE_B200_ENOMEM;
    }
}

static int care_b200_create_impl(const care_b200_options* opt, care_b200_ctx** out) {
    if (!opt || !out) return CARE_B200_EINVAL;
    *out = nullptr;
    auto c = std::make_unique<care_b200_ctx>();
    care_b200_ctx* ctx = c.get();
    ctx->opt = *opt;
    const int v = validate_options(ctx, *opt);
    if (v) return v;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (opt->device < 0 || opt->device >= ndev) return CARE_B200_EINVAL;
    CK(cudaSetDevice(opt->device), "cudaSetDevice");
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : ctx->ev) CK(cudaEventCreate(&e), "cudaEventCreate");
    CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    CK(cudaStreamCreateWithFlags(&ctx->copy_stream2, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& row : ctx->stage_ev)
        for (auto& e : row) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    float qw[256];
    quality_weights(qw);
    CK(cudaMemcpyToSymbol(c_qweight, qw, sizeof(qw)), "quality weights");
    ctx->threshold = results_per_map_threshold(opt->estimated_coverage);
    *out = c.release();
    return CARE_B200_OK;
}

int care_b200_destroy(care_b200_ctx* ctx) {
    if (!ctx) return CARE_B200_OK;
    cudaSetDevice(ctx->opt.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->sig_ev) if (e) cudaEventDestroy(e);
    ctx->sig_ev.clear();
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->copy_stream2) cudaStreamSynchronize(ctx->copy_stream2);
    for (auto& row : ctx->stage_ev)
        for (auto& e : row) if (e) cudaEventDestroy(e);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->copy_stream2) cudaStreamDestroy(ctx->copy_stream2);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CARE_B200_OK;
}

const char* care_b200_last_error(const care_b200_ctx* ctx) {
    return ctx ? ctx->err.c_str() : "no context";
}

static int care_b200_upload_reads_impl(care_b200_ctx* ctx, const uint32_t* packed, size_t pitch_ints,
                           const int32_t* lengths, const uint32_t* enc_quals, size_t qual_pitch_ints,
                           const uint32_t* ambiguous_ids, size_t num_ambiguous, uint32_t num_reads);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_upload_reads(care_b200_ctx* ctx, const uint32_t* packed, size_t pitch_ints,
                           const int32_t* lengths, const uint32_t* enc_quals, size_t qual_pitch_ints,
                           const uint32_t* ambiguous_ids, size_t num_ambiguous, uint32_t num_reads) {
    try {
        return care_b200_upload_reads_impl(ctx, packed, pitch_ints, lengths, enc_quals, qual_pitch_ints, ambiguous_ids, num_ambiguous, num_reads);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_upload_reads: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_upload_reads_impl(care_b200_ctx* ctx, const uint32_t* packed, size_t pitch_ints,
                           const int32_t* lengths, const uint32_t* enc_quals, size_t qual_pitch_ints,
                           const uint32_t* ambiguous_ids, size_t num_ambiguous, uint32_t num_reads) {
    if (!ctx) return CARE_B200_EINVAL;
    if (!packed || !lengths || num_reads == 0 || pitch_ints == 0) return fail(ctx, CARE_B200_EINVAL, "empty read storage");
    if (ctx->opt.paired_end && (num_reads % 2)) return fail(ctx, CARE_B200_EINVAL, "paired-end storage needs an even number of reads");
    int mx = 0;
    for (uint32_t i = 0; i < num_reads; i++) mx = std::max(mx, (int)lengths[i]);
    if (mx > kMaxLen) return fail(ctx, CARE_B200_ELIMIT, "reads longer than 256 bases are not supported");
    if ((size_t)(mx + 15) / 16 > pitch_ints) return fail(ctx, CARE_B200_EINVAL, "pitch_ints too small for the longest read");
    if (pitch_ints > (size_t)kMaxLen / 16) return fail(ctx, CARE_B200_EINVAL, "pitch_ints above 16 (256 bases)");
    if (enc_quals && ctx->opt.use_quality && qual_pitch_ints > (size_t)quality_ints(kMaxLen, ctx->opt.quality_bits))
        return fail(ctx, CARE_B200_EINVAL, "qual_pitch_ints above the words of 256 qualities");
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    ctx->n = num_reads;
    ctx->max_len = mx;
    ctx->seq_pitch = (int)pitch_ints;
    ctx->has_qual = enc_quals != nullptr && ctx->opt.use_quality;
    ctx->qual_pitch = ctx->has_qual ? (int)qual_pitch_ints : 0;
    if (ctx->has_qual && (size_t)quality_ints(mx, ctx->opt.quality_bits) > qual_pitch_ints)
        return fail(ctx, CARE_B200_EINVAL, "qual_pitch_ints too small for the longest read");
    // lengths, then the packed rows on the main stream, each chunk's whole
    // reads hashed (minhash signatures) as soon as its copy is enqueued; the
    // quality words upload on the copy stream meanwhile
    CK(cudaStreamSynchronize(ctx->stream), "upload");      // no earlier work still reads the storage
    CK(ctx->d_len.ensure((size_t)num_reads * 4), "alloc lengths");
    if (int rc = staged_upload(ctx, 0, ctx->d_len.p, lengths, (size_t)num_reads * 4, ctx->stream)) return rc;
    CK(ctx->d_seq.ensure((size_t)num_reads * pitch_ints * 4), "alloc reads");
    const int maps = ctx->num_maps ? ctx->num_maps : ctx->opt.num_maps;
    ctx->sigs_maps = 0;
    CK(ctx->d_sigs.ensure((size_t)num_reads * maps * 8), "alloc signatures");
    ctx->sig_used = 0;
    uint32_t hashed = 0;
    const size_t row_bytes = pitch_ints * 4;
    // copies on the copy stream; the main stream waits for each chunk's copy
    // and hashes its whole reads while the next chunks copy
    auto hash_chunk = [&](size_t end, cudaEvent_t done) -> int {
        if (done) CK(cudaStreamWaitEvent(ctx->stream, done, 0), "wait");
        const uint32_t whole = (uint32_t)std::min<size_t>(end / row_bytes, num_reads);
        const int rc = signatures_range(ctx, maps, hashed, whole);
        hashed = whole;
        return rc;
    };
    if (int rc = staged_upload(ctx, 0, ctx->d_seq.p, packed, (size_t)num_reads * row_bytes, ctx->copy_stream,
                               hash_chunk))
        return rc;
    ctx->sigs_maps = maps;
    if (ctx->has_qual) {
        CK(ctx->d_qual.ensure((size_t)num_reads * qual_pitch_ints * 4), "alloc qualities");
        if (int rc = staged_upload(ctx, 1, ctx->d_qual.p, enc_quals, (size_t)num_reads * qual_pitch_ints * 4,
                                   ctx->copy_stream2)) return rc;
    }
    ctx->h_len.assign(lengths, lengths + num_reads);
    ctx->h_ambig.assign(num_reads, 0);
    for (size_t i = 0; i < num_ambiguous; i++) {
        if (ambiguous_ids[i] >= num_reads) return fail(ctx, CARE_B200_EINVAL, "ambiguous id out of range");
        ctx->h_ambig[ambiguous_ids[i]] = 1;
    }
    CK(ctx->d_ambig.ensure(num_reads), "alloc ambiguous flags");
    CK(cudaMemcpyAsync(ctx->d_ambig.p, ctx->h_ambig.data(), num_reads, cudaMemcpyHostToDevice, ctx->stream), "upload ambiguous flags");
    CK(cudaStreamSynchronize(ctx->copy_stream), "upload");
    CK(cudaStreamSynchronize(ctx->copy_stream2), "upload");
    CK(cudaStreamSynchronize(ctx->stream), "upload");
    if (ctx->tables_ready && ctx->t_keys.size() && num_reads != ctx->tables_reads) ctx->tables_ready = false;
    ctx->r_valid = false;
    return CARE_B200_OK;
}

static int care_b200_upload_tables_impl(care_b200_ctx* ctx, int num_maps, const uint64_t* const* keys,
                            const uint32_t* const* offsets, const uint32_t* const* values,
                            const size_t* nkeys);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_upload_tables(care_b200_ctx* ctx, int num_maps, const uint64_t* const* keys,
                            const uint32_t* const* offsets, const uint32_t* const* values,
                            const size_t* nkeys) {
    try {
        return care_b200_upload_tables_impl(ctx, num_maps, keys, offsets, values, nkeys);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_upload_tables: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_upload_tables_impl(care_b200_ctx* ctx, int num_maps, const uint64_t* const* keys,
                            const uint32_t* const* offsets, const uint32_t* const* values,
                            const size_t* nkeys) {
    if (!ctx) return CARE_B200_EINVAL;
    if (num_maps < 1 || num_maps > kMaxMaps || !keys || !offsets || !values || !nkeys)
        return fail(ctx, CARE_B200_EINVAL, "invalid tables");
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    // open-addressing key index per map: capacity a power of two >= 2 keys
    std::vector<TableDesc> desc(num_maps);
    size_t total_slots = 0, total_values = 0;
    for (int m = 0; m < num_maps; m++) {
        size_t cap = 16;
        while (cap < 2 * nkeys[m]) cap <<= 1;
        desc[m].slot_base = total_slots;
        desc[m].value_base = total_values;
        desc[m].mask = (uint32_t)(cap - 1);
        total_slots += cap;
        total_values += nkeys[m] ? offsets[m][nkeys[m]] : 0;
    }
    if (total_values >= 0xFFFFFFFFull) return fail(ctx, CARE_B200_ELIMIT, "tables too large");
    std::vector<Slot> slots(total_slots, Slot{0, 0, 0});
    std::vector<uint32_t> vals(total_values);
    for (int m = 0; m < num_maps; m++) {
        Slot* s = slots.data() + desc[m].slot_base;
        const uint32_t mask = desc[m].mask;
        for (size_t i = 0; i < nkeys[m]; i++) {
            const uint32_t cnt = offsets[m][i + 1] - offsets[m][i];
            if (cnt == 0) continue;
            uint32_t pos = (uint32_t)host_murmur64(keys[m][i]) & mask;
            while (s[pos].count != 0) pos = (pos + 1) & mask;
            s[pos].key = keys[m][i];
            s[pos].offset = offsets[m][i];
            s[pos].count = cnt;
        }
        if (nkeys[m]) std::memcpy(vals.data() + desc[m].value_base, values[m], (size_t)offsets[m][nkeys[m]] * 4);
    }
    CK(ctx->d_slots.ensure(total_slots * sizeof(Slot)), "alloc slots");
    CK(ctx->d_values.ensure(std::max<size_t>(total_values, 1) * 4), "alloc values");
    CK(ctx->d_tdesc.ensure(num_maps * sizeof(TableDesc)), "alloc table descriptors");
    CK(cudaMemcpy(ctx->d_slots.p, slots.data(), total_slots * sizeof(Slot), cudaMemcpyHostToDevice), "upload slots");
    if (total_values) CK(cudaMemcpy(ctx->d_values.p, vals.data(), total_values * 4, cudaMemcpyHostToDevice), "upload values");
    CK(cudaMemcpy(ctx->d_tdesc.p, desc.data(), num_maps * sizeof(TableDesc), cudaMemcpyHostToDevice), "upload descriptors");
    ctx->num_maps = num_maps;
    ctx->t_keys.assign(num_maps, {});
    ctx->t_off.assign(num_maps, {});
    ctx->t_val.assign(num_maps, {});
    for (int m = 0; m < num_maps; m++) {
        ctx->t_keys[m].assign(keys[m], keys[m] + nkeys[m]);
        ctx->t_off[m].assign(offsets[m], offsets[m] + nkeys[m] + 1);
        const uint32_t nv = nkeys[m] ? offsets[m][nkeys[m]] : 0;
        ctx->t_val[m].assign(values[m], values[m] + nv);
    }
    ctx->tables_ready = true;
    ctx->tables_reads = ctx->n;
    return CARE_B200_OK;
}

static int care_b200_build_tables_impl(care_b200_ctx* ctx);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_build_tables(care_b200_ctx* ctx) {
    try {
        return care_b200_build_tables_impl(ctx);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_build_tables: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_build_tables_impl(care_b200_ctx* ctx) {
    if (!ctx) return CARE_B200_EINVAL;
    if (ctx->n == 0) return fail(ctx, CARE_B200_ESTATE, "no reads uploaded");
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    const int h = ctx->opt.num_maps;
    ctx->num_maps = h;
    DevOptions o = make_dev_options(ctx);
    DevReads r = make_dev_reads(ctx);
    // signatures of all reads on the device (insert, ordinaryminhasher.hpp:376-426),
    // kept resident for the candidate stage
    if (ctx->sigs_maps != h)
        if (int rc = compute_signatures(ctx, h)) return rc;
    {
        // grouping on the device: radix sort, runs, kept keys, slots
        DeviceTables t = build_tables_device(ctx->d_sigs.as<unsigned long long>(), ctx->n, h,
                                             ctx->opt.kmerlength, ctx->threshold, ctx->stream);
        if (t.error == cudaSuccess) {
            // host copies for care_b200_get_table
            std::vector<unsigned long long> keys(t.nkeys);
            std::vector<uint32_t> koff(t.nkeys), vals(t.nvalues);
            if (t.nkeys) {
                CK(cudaMemcpyAsync(keys.data(), t.keys.p, (size_t)t.nkeys * 8, cudaMemcpyDeviceToHost, ctx->stream), "tables");
                CK(cudaMemcpyAsync(koff.data(), t.key_off.p, (size_t)t.nkeys * 4, cudaMemcpyDeviceToHost, ctx->stream), "tables");
            }
            if (t.nvalues)
                CK(cudaMemcpyAsync(vals.data(), t.values.p, (size_t)t.nvalues * 4, cudaMemcpyDeviceToHost, ctx->stream), "tables");
            CK(cudaStreamSynchronize(ctx->stream), "tables");
            ctx->num_maps = h;
            ctx->t_keys.assign(h, {});
            ctx->t_off.assign(h, {});
            ctx->t_val.assign(h, {});
            for (int m = 0; m < h; m++) {
                const uint32_t f = t.map_first[m], c = t.map_keys[m], vb = t.map_vbase[m], vc = t.map_vcount[m];
                ctx->t_keys[m].assign(keys.begin() + f, keys.begin() + f + c);
                auto& off = ctx->t_off[m];
                off.resize(c + 1);
                for (uint32_t i = 0; i < c; i++) off[i] = koff[f + i] - vb;
                off[c] = vc;
                ctx->t_val[m].assign(vals.begin() + vb, vals.begin() + vb + vc);
            }
            const size_t ns = t.total_slots, nv = std::max<size_t>(t.nvalues, 1);
            ctx->d_slots.adopt(t.slots.release(), ns * sizeof(Slot));
            ctx->d_values.adopt(t.values.release(), nv * 4);
            ctx->d_tdesc.adopt(t.desc.release(), (size_t)h * sizeof(TableDesc));
            ctx->tables_ready = true;
            ctx->tables_reads = ctx->n;
            return CARE_B200_OK;
        }
        // only a composite key wider than 64 bits (2k + log2(maps)) sends the
        // grouping to the host; any other failure is an error
        if (t.error != cudaErrorInvalidValue) return cuda_fail(ctx, t.error, "table build on the device");
        cudaGetLastError();
    }
    std::vector<uint64_t> sig((size_t)ctx->n * h);
    CK(cudaMemcpyAsync(sig.data(), ctx->d_sigs.p, (size_t)ctx->n * h * 8, cudaMemcpyDeviceToHost, ctx->stream), "signatures");
    CK(cudaStreamSynchronize(ctx->stream), "signatures");
    // group per map: values of one key ascending, buckets with fewer than 2
    // or more than threshold values cleared (groupbykey.hpp:99-249)
    const uint32_t n = ctx->n;
    const int thr = ctx->threshold;
    std::vector<std::vector<uint64_t>> K(h);
    std::vector<std::vector<uint32_t>> O(h), Vv(h);
    auto build = [&](int m0, int m1) {
        std::vector<std::pair<uint64_t, uint32_t>> kv(n);
        for (int m = m0; m < m1; m++) {
            for (uint32_t i = 0; i < n; i++) kv[i] = {sig[(size_t)i * h + m], i};
            std::sort(kv.begin(), kv.end());
            auto& keys = K[m]; auto& off = O[m]; auto& val = Vv[m];
            off.push_back(0);
            for (uint32_t i = 0; i < n;) {
                uint32_t e = i;
                while (e < n && kv[e].first == kv[i].first) e++;
                const uint32_t c = e - i;
                if (c >= 2 && (int)c <= thr) {
                    keys.push_back(kv[i].first);
                    for (uint32_t x = i; x < e; x++) val.push_back(kv[x].second);
                    off.push_back((uint32_t)val.size());
                }
                i = e;
            }
        }
    };
    unsigned nt = ctx->opt.threads > 0 ? (unsigned)ctx->opt.threads : std::thread::hardware_concurrency();
    nt = std::max(1u, std::min<unsigned>(nt, (unsigned)h));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) th.emplace_back(build, (int)(h * t / nt), (int)(h * (t + 1) / nt));
    for (auto& x : th) x.join();
    std::vector<const uint64_t*> kp(h);
    std::vector<const uint32_t*> op(h), vp(h);
    std::vector<size_t> nk(h);
    for (int m = 0; m < h; m++) { kp[m] = K[m].data(); op[m] = O[m].data(); vp[m] = Vv[m].data(); nk[m] = K[m].size(); }
    return care_b200_upload_tables(ctx, h, kp.data(), op.data(), vp.data(), nk.data());
}

static int care_b200_get_table_impl(care_b200_ctx* ctx, int map, const uint64_t** keys, const uint32_t** offsets,
                        const uint32_t** values, size_t* nkeys);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_get_table(care_b200_ctx* ctx, int map, const uint64_t** keys, const uint32_t** offsets,
                        const uint32_t** values, size_t* nkeys) {
    try {
        return care_b200_get_table_impl(ctx, map, keys, offsets, values, nkeys);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_get_table: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_get_table_impl(care_b200_ctx* ctx, int map, const uint64_t** keys, const uint32_t** offsets,
                        const uint32_t** values, size_t* nkeys) {
    if (!ctx) return CARE_B200_EINVAL;
    if (!ctx->tables_ready || map < 0 || map >= ctx->num_maps) return fail(ctx, CARE_B200_EINVAL, "no such table");
    *keys = ctx->t_keys[map].data();
    *offsets = ctx->t_off[map].data();
    *values = ctx->t_val[map].data();
    *nkeys = ctx->t_keys[map].size();
    return CARE_B200_OK;
}

}  // extern "C"

namespace {

// ---- launch dispatch of the tuned stage mappings ----

struct AlignArgs {
    DevOptions o; DevReads r; uint32_t first;
    const uint32_t* cand_ids; const uint32_t* cand_anchor; const uint32_t* seg_off; const uint32_t* seg_cnt;
    const unsigned long long* total; unsigned long long cap; const int* status; AlignRes* out;
    unsigned long long* words; const uint32_t* pair_order;
    const uint2* work; const unsigned int* work_n;
    unsigned long long* run_words;             // non-null: the statistics form, counting words run
    bool warp;                                 // k_align_warp: a warp per work item
    int sms;
    const uint2* cls;                          // one length class of the pairs (pair_order = the class list)
};

template <int B, int NW, bool CNT>
cudaError_t align_go(const AlignArgs& a, cudaStream_t st) {
    if (a.warp) {
        // persistent: the resident blocks' warps stride over the work items
        int nb = 0;
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_align_warp<B, NW, CNT>, B, 0);
        if (e != cudaSuccess) return e;
        const unsigned long long need = (a.cap + B / 32 - 1) / (B / 32);
        const unsigned grid = (unsigned)std::max<unsigned long long>(
            1, std::min<unsigned long long>(need, (unsigned long long)a.sms * std::max(nb, 1)));
        k_align_warp<B, NW, CNT><<<grid, B, 0, st>>>(a.o, a.r, a.first, a.cand_ids, a.cand_anchor, a.seg_off,
                                                     a.seg_cnt, a.total, a.cap, a.status, a.out, a.words,
                                                     a.pair_order, a.work, a.work_n, a.run_words);
        return cudaGetLastError();
    }
    const unsigned long long blocks = (a.cap + B - 1) / B;
    if (a.cls) {        // a length class: resident blocks striding over its pairs
        int nb = 0;
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_align_class<B, NW, CNT>, B, 0);
        if (e != cudaSuccess) return e;
        const unsigned grid = (unsigned)std::max<unsigned long long>(
            1, std::min<unsigned long long>(blocks, (unsigned long long)a.sms * std::max(nb, 1)));
        k_align_class<B, NW, CNT><<<grid, B, 0, st>>>(a.o, a.r, a.first, a.cand_ids, a.cand_anchor, a.seg_off,
                                                      a.seg_cnt, a.total, a.cap, a.status, a.out, a.words,
                                                      a.pair_order, a.cls, a.run_words);
        return cudaGetLastError();
    }
    k_align<B, NW, CNT><<<(unsigned)blocks, B, 0, st>>>(a.o, a.r, a.first, a.cand_ids, a.cand_anchor, a.seg_off,
                                                        a.seg_cnt, a.total, a.cap, a.status, a.out, a.words,
                                                        a.pair_order, a.work, a.work_n, a.run_words);
    return cudaGetLastError();
}

cudaError_t align_dispatch(int block, int nw, const AlignArgs& a, cudaStream_t st) {
#define AL(B, C)                                        \
    if (nw <= 4) return align_go<B, 4, C>(a, st);       \
    if (nw <= 5) return align_go<B, 5, C>(a, st);       \
    if (nw <= 6) return align_go<B, 6, C>(a, st);       \
    return align_go<B, 8, C>(a, st);
    if (a.run_words) {
        if (block == 256) { AL(256, true) }
        AL(128, true)
    }
    if (block == 256) { AL(256, false) }
    AL(128, false)
#undef AL
}

struct MsaArgs {
    DevOptions o; DevReads r; uint32_t first, count;
    const uint32_t* order; unsigned int* cursor;
    const uint32_t* cand_ids; const uint32_t* seg_off; const uint32_t* seg_cnt; const AlignRes* ares;
    CandRec* recs; MsaOut out; int* status; size_t smem;
    bool queue; int sms; int grid;             // grid: resident CTAs of the queue form (prepare)
    int jb;                                    // 32-column blocks per warp
};

// prepare (host only: attributes, occupancy) or launch one MSA variant
template <int B, int QB, bool E>
cudaError_t msa_go(MsaArgs& a, bool prepare, cudaStream_t st) {
    if (prepare) {
        cudaError_t e = cudaFuncSetAttribute(k_msa<B, QB, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_msa_queue<B, QB, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.smem);
        int nb = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_msa_queue<B, QB, E>, B, a.smem);
        a.grid = (int)std::min<uint64_t>(a.count, (uint64_t)a.sms * (uint64_t)std::max(nb, 1));
        return e;
    }
    if (a.queue)
        k_msa_queue<B, QB, E><<<a.grid, B, a.smem, st>>>(a.o, a.r, a.first, a.count, a.jb, a.order, a.cursor,
                                                        a.cand_ids, a.seg_off, a.seg_cnt, a.ares, a.recs, a.out,
                                                        a.status);
    else
        k_msa<B, QB, E><<<a.count, B, a.smem, st>>>(a.o, a.r, a.first, a.count, a.jb, a.order, a.cand_ids,
                                                    a.seg_off, a.seg_cnt, a.ares, a.recs, a.out, a.status);
    return cudaGetLastError();
}

// qb: the quality encoding the column sums read (0 when qualities are unused)
cudaError_t msa_dispatch(int warps, int qb, bool emit, MsaArgs& a, bool prepare, cudaStream_t st) {
#define MS(B, Q) return emit ? msa_go<B, Q, true>(a, prepare, st) : msa_go<B, Q, false>(a, prepare, st);
    if (warps == 8) {
        switch (qb) { case 0: MS(256, 0) case 1: MS(256, 1) case 2: MS(256, 2) default: MS(256, 8) }
    }
    switch (qb) { case 0: MS(128, 0) case 1: MS(128, 1) case 2: MS(128, 2) default: MS(128, 8) }
#undef MS
}

// Runs the stages for anchors [first, first+count) into the device output
// buffers; grows the arenas and repeats on overflow. With tune.graph each
// attempt's launches, memsets and copies are captured and replayed as one
// CUDA graph (the instantiated graph is updated in place for the next batch).
int run_batch(care_b200_ctx* ctx, uint32_t first, uint32_t count, bool timed) {
    const DevOptions o = make_dev_options(ctx);
    const DevReads r = make_dev_reads(ctx);
    const care_b200_tuning& tu = ctx->tune;
    const int h = ctx->num_maps;
    // shared hash set for de-duplication: > num_maps * threshold entries
    const size_t tmax = (size_t)h * ctx->threshold;
    int set_log2 = 6;                 // at least 64 entries: the set and the sort pad to 64 and 32
    while ((size_t)1 << set_log2 < (tmax * 4 + 2) / 3 + 1) set_log2++;
    const int groups = kCandBlock / h;
    const size_t cand_smem = CandSmem::total(ctx->max_len, groups, h, ctx->seq_pitch, 1 << set_log2);
    if (cand_smem > 227 * 1024) return fail(ctx, CARE_B200_ELIMIT, "num_maps * threshold too large for the de-duplication set");
    if (ctx->sms == 0) CK(cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->opt.device), "attr");
    // the main candidate pass uses a set of at most 2^cand_set_log2 entries
    // (high occupancy); anchors with more unique ids than half of it are
    // redone by k_candidates_spill with the full set
    const bool spill = set_log2 > tu.cand_set_log2;
    const int set_log2_main = spill ? tu.cand_set_log2 : set_log2;
    const size_t cand_smem_main = CandSmem::total(ctx->max_len, groups, h, ctx->seq_pitch, 1 << set_log2_main);
    CK(cudaFuncSetAttribute(k_candidates<kCandBlock>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)cand_smem_main), "smem attr");
    int spill_grid = 0;
    if (spill) {
        CK(cudaFuncSetAttribute(k_candidates_spill<kCandBlock>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)cand_smem), "smem attr");
        int nb = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_candidates_spill<kCandBlock>, kCandBlock, cand_smem),
           "occupancy");
        spill_grid = ctx->sms * std::max(nb, 1);
        CK(ctx->d_spill.ensure((size_t)count * 4), "alloc");
    }

    CK(ctx->d_seg_off.ensure((size_t)count * 4), "alloc");
    CK(ctx->d_seg_cnt.ensure((size_t)count * 4), "alloc");
    CK(ctx->d_counters.ensure(128), "alloc");
    CK(ctx->d_status.ensure(16), "alloc");
    CK(ctx->d_st.ensure(count), "alloc");
    CK(ctx->d_ned.ensure((size_t)count * 4), "alloc");
    CK(ctx->d_oseq.ensure((size_t)count * ctx->max_len), "alloc");
    CK(ctx->h_small.ensure(96), "alloc");
    if (tu.msa_order) {
        CK(ctx->d_order.ensure((size_t)count * 4), "alloc");
        CK(ctx->d_bins.ensure(kLptBins * 4), "alloc");
    }
    {   // the pairs per anchor seen last, with a margin (96 before the first call)
        const unsigned long long want = std::min<unsigned long long>(
            kMaxBatchPairs, (unsigned long long)((double)count * ctx->pairs_per_anchor * 1.1) + 1024);
        if (ctx->cand_cap < want) ctx->cand_cap = want;
    }
    if (ctx->corr_cap == 0) ctx->corr_cap = ctx->opt.correct_candidates ? (unsigned long long)count * 16 + 1024 : 1024;
    const bool emit = o.clf_mode != 0;
    if (emit) {
        if (ctx->feat_cap < (unsigned long long)count / 2 + 4096) ctx->feat_cap = (unsigned long long)count / 2 + 4096;
        CK(ctx->d_touched.ensure(count), "alloc");
        CK(ctx->d_mlp_err.ensure(16), "alloc");
    }
    // widest possible MSA: La + 2*Lmax - 2*minoverlap(La), maximised over La
    int maxcols = 1;
    for (int la = 1; la <= ctx->max_len; ++la) {
        const int lo = (int)((float)la * ctx->opt.min_overlap_ratio);
        const int mo = std::max(ctx->opt.min_overlap, lo);
        maxcols = std::max(maxcols, la + 2 * ctx->max_len - 2 * std::min(mo, ctx->max_len));
    }
    const int warps = tu.msa_warps == 8 ? 8 : 4;
    const int jb = (maxcols + 32 * warps - 1) / (32 * warps);
    const int nw = (ctx->max_len + 31) / 32;           // bit-plane width: 32-base words of the longest read
    // length classes of the alignment (not with mirror pairs, whose work list pairs equal lengths)
    const bool classes = tu.align_classes != 0 && tu.pair_mirror == 0;
    if (classes) CK(ctx->d_cls.ensure(64), "alloc");
    const int qb = ctx->has_qual ? ctx->opt.quality_bits : 0;
    const size_t msmem = msa_smem_bytes(ctx->max_len, ctx->seq_pitch, ctx->has_qual ? ctx->qual_pitch : 0, qb, emit,
                                        32 * jb * warps);

    for (int attempt = 0; attempt < 8; ++attempt) {
        const unsigned long long cap = ctx->cand_cap;
        CK(ctx->d_cand_ids.ensure(cap * 4), "alloc candidates");
        CK(ctx->d_cand_anchor.ensure(cap * 4), "alloc candidates");
        CK(ctx->d_ares.ensure(cap * sizeof(AlignRes)), "alloc alignments");
        CK(ctx->d_recs.ensure(cap * sizeof(CandRec)), "alloc records");
        if (tu.pair_order) CK(ctx->d_pair_order.ensure(cap * 4), "alloc pair order");
        if (tu.pair_mirror) CK(ctx->d_pair_work.ensure(cap * 8), "alloc mirror work list");
        if (classes) CK(ctx->d_pair_class.ensure(cap * 4), "alloc pair classes");
        const unsigned long long ccap = ctx->corr_cap;
        CK(ctx->d_cid.ensure(ccap * 4), "alloc");
        CK(ctx->d_canc.ensure(ccap * 4), "alloc");
        CK(ctx->d_cshift.ensure(ccap * 4), "alloc");
        CK(ctx->d_cue.ensure(ccap), "alloc");
        CK(ctx->d_cseq.ensure(ccap * ctx->max_len), "alloc");
        const unsigned long long fcap = ctx->feat_cap;
        if (emit) {
            CK(ctx->d_fx.ensure(fcap * kNumFeatures * 4), "alloc decision rows");
            CK(ctx->d_fread.ensure(fcap * 4), "alloc decision rows");
            CK(ctx->d_fmeta.ensure(fcap * 4), "alloc decision rows");
            CK(ctx->d_flogit.ensure(fcap * 4), "alloc decision rows");
        }
        unsigned long long* counters = ctx->d_counters.as<unsigned long long>();
        int* status = ctx->d_status.as<int>();

        MsaOut mo;
        mo.status = ctx->d_st.as<uint8_t>();
        mo.nedits = ctx->d_ned.as<int32_t>();
        mo.seq = ctx->d_oseq.as<char>();
        mo.corr_id = ctx->d_cid.as<uint32_t>();
        mo.corr_anchor = ctx->d_canc.as<uint32_t>();
        mo.corr_shift = ctx->d_cshift.as<int32_t>();
        mo.corr_use_edits = ctx->d_cue.as<uint8_t>();
        mo.corr_seq = ctx->d_cseq.as<char>();
        mo.corr_count = counters + 1;
        mo.corr_cap = ccap;
        mo.feat = emit ? ctx->d_fx.as<float>() : nullptr;
        mo.feat_read = emit ? ctx->d_fread.as<uint32_t>() : nullptr;
        mo.feat_meta = emit ? ctx->d_fmeta.as<uint32_t>() : nullptr;
        mo.feat_count = counters + 2;
        mo.feat_cap = emit ? fcap : 0;
        mo.elem_count = counters + 5;
        mo.rebuild_count = counters + 9;             // counters 9 and 10

        AlignArgs aa{o, r, first, ctx->d_cand_ids.as<uint32_t>(), ctx->d_cand_anchor.as<uint32_t>(),
                     ctx->d_seg_off.as<uint32_t>(), ctx->d_seg_cnt.as<uint32_t>(), counters, cap, status,
                     ctx->d_ares.as<AlignRes>(), counters + 3,
                     tu.pair_order ? ctx->d_pair_order.as<uint32_t>() : nullptr,
                     tu.pair_mirror ? ctx->d_pair_work.as<uint2>() : nullptr,
                     reinterpret_cast<const unsigned int*>(counters + 6),
                     ctx->count_words ? counters + 8 : nullptr, tu.align_warp != 0, ctx->sms, nullptr};
        MsaArgs ma{o, r, first, count, tu.msa_order ? ctx->d_order.as<uint32_t>() : nullptr,
                   reinterpret_cast<unsigned int*>(counters + 4), ctx->d_cand_ids.as<uint32_t>(),
                   ctx->d_seg_off.as<uint32_t>(), ctx->d_seg_cnt.as<uint32_t>(), ctx->d_ares.as<AlignRes>(),
                   ctx->d_recs.as<CandRec>(), mo, status, msmem, tu.msa_queue != 0, ctx->sms, 0, jb};
        CK(msa_dispatch(warps, qb, emit, ma, true, ctx->stream), "MSA launch setup");

        cudaStream_t st = ctx->stream;
        const bool graph = tu.graph != 0;
        auto mark = [&](int k) -> cudaError_t {
            if (!timed) return cudaSuccess;
            return graph ? cudaEventRecordWithFlags(ctx->ev[k], st, cudaEventRecordExternal)
                         : cudaEventRecord(ctx->ev[k], st);
        };
        // every operation of one attempt, in stream order
        int launches = 0;                     // kernels of this library enqueued by the attempt
        auto enqueue = [&]() -> int {
            launches = 0;
#define EQ(call, where) do { const cudaError_t e_ = (call); if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); } while (0)
            EQ(cudaMemsetAsync(counters, 0, 128, st), "memset");
            EQ(cudaMemsetAsync(status, 0, 16, st), "memset");
            // rows of anchors that are not corrected read as zero bytes
            EQ(cudaMemsetAsync(ctx->d_oseq.p, 0, (size_t)count * ctx->max_len, st), "memset");
            if (emit) {
                EQ(cudaMemsetAsync(ctx->d_touched.p, 0, count, st), "memset");
                EQ(cudaMemsetAsync(ctx->d_mlp_err.p, 0, 16, st), "memset");
            }
            EQ(mark(0), "event");
            unsigned int* spill_n = reinterpret_cast<unsigned int*>(counters + 7);
            k_candidates<kCandBlock><<<count, kCandBlock, cand_smem_main, st>>>(
                o, r, ctx->d_tdesc.as<TableDesc>(), ctx->d_slots.as<Slot>(), ctx->d_values.as<uint32_t>(),
                ctx->d_sigs.as<unsigned long long>(), first, count, set_log2_main,
                spill ? ctx->d_spill.as<uint32_t>() : nullptr, spill ? spill_n : nullptr,
                ctx->d_cand_ids.as<uint32_t>(), ctx->d_cand_anchor.as<uint32_t>(),
                ctx->d_seg_off.as<uint32_t>(), ctx->d_seg_cnt.as<uint32_t>(), counters, cap, status);
            EQ(cudaGetLastError(), "k_candidates");
            ++launches;
            if (spill) {
                k_candidates_spill<kCandBlock><<<spill_grid, kCandBlock, cand_smem, st>>>(
                    o, r, ctx->d_tdesc.as<TableDesc>(), ctx->d_slots.as<Slot>(), ctx->d_values.as<uint32_t>(),
                    ctx->d_sigs.as<unsigned long long>(), first, set_log2, ctx->d_spill.as<uint32_t>(), spill_n,
                    ctx->d_cand_ids.as<uint32_t>(), ctx->d_cand_anchor.as<uint32_t>(),
                    ctx->d_seg_off.as<uint32_t>(), ctx->d_seg_cnt.as<uint32_t>(), counters, cap, status);
                EQ(cudaGetLastError(), "k_candidates_spill");
                ++launches;
            }
            EQ(mark(1), "event");
            if (tu.pair_order) {
                k_pair_order<<<count, 128, 0, st>>>(r, ctx->d_cand_ids.as<uint32_t>(), ctx->d_seg_off.as<uint32_t>(),
                                                    ctx->d_seg_cnt.as<uint32_t>(), count, status,
                                                    ctx->d_pair_order.as<uint32_t>());
                EQ(cudaGetLastError(), "k_pair_order");
                ++launches;
            }
            if (tu.pair_mirror) {
                k_pair_mirror<256><<<(unsigned)((cap + 255) / 256), 256, 0, st>>>(
                    r, first, count, ctx->d_cand_ids.as<uint32_t>(), ctx->d_cand_anchor.as<uint32_t>(),
                    ctx->d_seg_off.as<uint32_t>(), ctx->d_seg_cnt.as<uint32_t>(), counters, cap, status,
                    tu.pair_order ? ctx->d_pair_order.as<uint32_t>() : nullptr, ctx->d_pair_work.as<uint2>(),
                    reinterpret_cast<unsigned int*>(counters + 6));
                EQ(cudaGetLastError(), "k_pair_mirror");
                ++launches;
            }
            if (classes) {
                // pairs by length class, then one alignment launch per class
                const unsigned g = (unsigned)ctx->sms * 8;
                uint2* cls = ctx->d_cls.as<uint2>();
                unsigned int* cursor = reinterpret_cast<unsigned int*>(cls + kAlignClasses);
                const uint32_t* order_in = tu.pair_order ? ctx->d_pair_order.as<uint32_t>() : nullptr;
                EQ(cudaMemsetAsync(ctx->d_cls.p, 0, 64, st), "memset");
                k_pair_class_count<<<g, 256, 0, st>>>(r, first, ctx->d_cand_ids.as<uint32_t>(),
                                                      ctx->d_cand_anchor.as<uint32_t>(), counters, cap, status,
                                                      order_in, cls);
                k_pair_class_offsets<<<1, 32, 0, st>>>(cls, cursor);
                k_pair_class_scatter<<<g, 256, 0, st>>>(r, first, ctx->d_cand_ids.as<uint32_t>(),
                                                        ctx->d_cand_anchor.as<uint32_t>(), counters, cap, status,
                                                        order_in, cursor, ctx->d_pair_class.as<uint32_t>());
                EQ(cudaGetLastError(), "pair classes");
                launches += 3;
                for (int c = 0; c < kAlignClasses; ++c) {
                    if (align_class_width(c) > std::max(nw, 4) && c > 0 && align_class_width(c - 1) >= nw) break;
                    AlignArgs ac = aa;
                    ac.pair_order = ctx->d_pair_class.as<uint32_t>();
                    ac.cls = cls + c;
                    EQ(align_dispatch(tu.align_block, align_class_width(c), ac, st), "k_align");
                    ++launches;
                }
            } else {
                EQ(align_dispatch(tu.align_block, nw, aa, st), "k_align");
                ++launches;
            }
            EQ(mark(2), "event");
            if (tu.msa_order) {
                const unsigned g = (unsigned)std::min<uint64_t>(((uint64_t)count + 255) / 256, (uint64_t)ctx->sms * 8);
                EQ(cudaMemsetAsync(ctx->d_bins.p, 0, kLptBins * 4, st), "memset");
                k_lpt_hist<<<g, 256, 0, st>>>(ctx->d_seg_cnt.as<uint32_t>(), count, ctx->d_bins.as<unsigned int>());
                k_lpt_scan<<<1, 1024, 0, st>>>(ctx->d_bins.as<unsigned int>());
                k_lpt_scatter<<<g, 256, 0, st>>>(ctx->d_seg_cnt.as<uint32_t>(), count, ctx->d_bins.as<unsigned int>(),
                                                 ctx->d_order.as<uint32_t>());
                EQ(cudaGetLastError(), "LPT order");
                launches += 3;
            }
            EQ(msa_dispatch(warps, qb, emit, ma, false, st), "k_msa");
            ++launches;
            EQ(mark(3), "event");
            if (o.clf_mode == 2) {
                // the network decides the batch's decision columns (row count
                // read on the device), then the changed anchors' edit counts
                EQ(mlp_infer(ctx->d_mlp.as<float>(), ctx->d_fx.as<float>(), fcap, counters + 2,
                             ctx->d_flogit.as<float>(), ctx->d_mlp_err.as<int>(), st), "k_mlp_infer");
                k_clf_apply<<<ctx->sms * 4, 256, 0, st>>>(ctx->d_fread.as<uint32_t>(), ctx->d_fmeta.as<uint32_t>(),
                                                          ctx->d_flogit.as<float>(), counters + 2, fcap, first,
                                                          ctx->max_len, ctx->d_oseq.as<char>(),
                                                          ctx->d_touched.as<uint8_t>());
                EQ(cudaGetLastError(), "k_clf_apply");
                k_clf_recount<<<(count + 7) / 8, 256, 0, st>>>(r, first, count, ctx->d_touched.as<uint8_t>(),
                                                               ctx->d_oseq.as<char>(), ctx->d_st.as<uint8_t>(),
                                                               ctx->d_ned.as<int32_t>());
                EQ(cudaGetLastError(), "k_clf_recount");
                launches += 3;                   // inference, verdicts, recount
            }
            EQ(mark(4), "event");
            EQ(cudaMemcpyAsync(ctx->h_small.p, counters, 88, cudaMemcpyDeviceToHost, st), "counters");
            EQ(cudaMemcpyAsync(ctx->h_small.as<char>() + 88, status, 4, cudaMemcpyDeviceToHost, st), "status");
            if (o.clf_mode == 2)
                EQ(cudaMemcpyAsync(ctx->h_small.as<char>() + 92, ctx->d_mlp_err.p, 4, cudaMemcpyDeviceToHost, st), "status");
#undef EQ
            return CARE_B200_OK;
        };
        if (graph) {
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
            const int rc = enqueue();
            cudaGraph_t g = nullptr;
            const cudaError_t ee = cudaStreamEndCapture(st, &g);
            if (rc) { if (g) cudaGraphDestroy(g); return rc; }
            CK(ee, "end capture");
            cudaError_t ge = cudaErrorUnknown;
            if (ctx->gexec) {
                cudaGraphExecUpdateResultInfo info;
                ge = cudaGraphExecUpdate(ctx->gexec, g, &info);
                if (ge != cudaSuccess) { cudaGetLastError(); cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
            }
            if (!ctx->gexec) ge = cudaGraphInstantiate(&ctx->gexec, g, 0);
            cudaGraphDestroy(g);
            CK(ge, "instantiate graph");
            CK(cudaGraphLaunch(ctx->gexec, st), "graph launch");
        } else {
            if (int rc = enqueue()) return rc;
        }
        CK(cudaStreamSynchronize(st), "batch");
        ctx->r_launches += launches;
        const unsigned long long used = ctx->h_small.as<unsigned long long>()[0];
        const unsigned long long corr = ctx->h_small.as<unsigned long long>()[1];
        const unsigned long long nfeat = ctx->h_small.as<unsigned long long>()[2];
        const unsigned long long words = ctx->h_small.as<unsigned long long>()[3];
        const unsigned long long elems = ctx->h_small.as<unsigned long long>()[5];
        const unsigned int spilled = ctx->h_small.as<unsigned int>()[14];     // counters + 7
        const unsigned long long run_words = ctx->h_small.as<unsigned long long>()[8];
        const unsigned long long rb_elems = ctx->h_small.as<unsigned long long>()[9];
        const unsigned long long rb_anchors = ctx->h_small.as<unsigned long long>()[10];
        const int stw = *(int*)(ctx->h_small.as<char>() + 88);
        if (stw & kStatusColumns) return fail(ctx, CARE_B200_ELIMIT, "MSA wider than the kernel's column capacity");
        bool again = false;
        if ((stw & kStatusCandOverflow) || used > cap) {
            // pair indices and segment offsets are 32-bit
            if (used + used / 8 + 1024 > kMaxBatchPairs)
                return fail(ctx, CARE_B200_ELIMIT, "more than 2^32-1 candidate pairs in one batch: set a smaller batch_size");
            ctx->cand_cap = used + used / 8 + 1024;
            again = true;
        }
        if ((stw & kStatusCorrOverflow) || corr > ccap) { ctx->corr_cap = corr + corr / 8 + 1024; again = true; }
        if (emit && ((stw & kStatusFeatOverflow) || nfeat > fcap)) { ctx->feat_cap = nfeat + nfeat / 8 + 4096; again = true; }
        if (again) continue;
        if (o.clf_mode == 2 && *(int*)(ctx->h_small.as<char>() + 92))
            return fail(ctx, CARE_B200_ECUDA, "tensor-core completion wait ran out");
        if (timed) {
            float a = 0, b = 0, c = 0, d = 0;
            cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
            cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
            cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]);
            cudaEventElapsedTime(&d, ctx->ev[3], ctx->ev[4]);
            ctx->stage_ms[0] += a; ctx->stage_ms[1] += b; ctx->stage_ms[2] += c; ctx->stage_ms[3] += d;
            ctx->last_ms += a + b + c + d;
        }
        if (emit && ctx->collect && nfeat) {
            const size_t b0 = ctx->r_fread.size();
            ctx->r_fx.resize((b0 + nfeat) * kNumFeatures);
            ctx->r_fread.resize(b0 + nfeat);
            ctx->r_fmeta.resize(b0 + nfeat);
            CK(cudaMemcpyAsync(ctx->r_fx.data() + b0 * kNumFeatures, ctx->d_fx.p, nfeat * kNumFeatures * 4, cudaMemcpyDeviceToHost, st), "rows");
            CK(cudaMemcpyAsync(ctx->r_fread.data() + b0, ctx->d_fread.p, nfeat * 4, cudaMemcpyDeviceToHost, st), "rows");
            CK(cudaMemcpyAsync(ctx->r_fmeta.data() + b0, ctx->d_fmeta.p, nfeat * 4, cudaMemcpyDeviceToHost, st), "rows");
            if (o.clf_mode == 2) {
                ctx->r_flogit.resize(b0 + nfeat);
                CK(cudaMemcpyAsync(ctx->r_flogit.data() + b0, ctx->d_flogit.p, nfeat * 4, cudaMemcpyDeviceToHost, st), "rows");
            }
            CK(cudaStreamSynchronize(st), "rows");
        }
        ctx->r_ncand += corr;
        ctx->r_pairs += used;
        ctx->r_words += words;
        ctx->r_elems += elems;
        ctx->r_rb_elems += rb_elems;
        ctx->r_rb_anchors += rb_anchors;
        ctx->r_spilled += spilled;
        ctx->r_run_words += run_words;
        return (int)std::min<unsigned long long>(corr, 0x7fffffff);
    }
    return fail(ctx, CARE_B200_ENOMEM, "arena growth did not converge");
}

// Anchors per batch when the caller leaves it to the library: as many as half
// of the free device memory holds at the pairs per anchor seen last (96 before
// the first call) -- one batch for most read sets, so that every candidate is
// an anchor of the same batch (mirror pairs) and nothing is launched twice --
// at least 2^20, and few enough for 32-bit pair indices with room to grow.
uint32_t auto_batch(care_b200_ctx* ctx, uint32_t count) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); return 1u << 21; }
    // the batch scratch this context already holds is reused, not added
    for (const DBuf* d : {&ctx->d_seg_off, &ctx->d_seg_cnt, &ctx->d_cand_ids, &ctx->d_cand_anchor, &ctx->d_ares,
                          &ctx->d_recs, &ctx->d_st, &ctx->d_ned, &ctx->d_oseq, &ctx->d_cid, &ctx->d_canc,
                          &ctx->d_cshift, &ctx->d_cue, &ctx->d_cseq, &ctx->d_order, &ctx->d_pair_order,
                          &ctx->d_pair_work, &ctx->d_fx, &ctx->d_fread, &ctx->d_fmeta, &ctx->d_flogit,
                          &ctx->d_touched, &ctx->d_spill})
        free_b += d->bytes;
    const double ppa = ctx->pairs_per_anchor;
    const double L = ctx->max_len;
    double per_anchor = ppa * (4 + 4 + sizeof(AlignRes) + sizeof(CandRec) + 8 + 4)   // ids, anchors, alignments,
                        + 2 * L + 64;                                             // records, work, order; rows
    if (ctx->opt.correct_candidates) per_anchor += 16 * (13 + L);
    if (ctx->opt.correction_type == 1) per_anchor += 0.5 * (kNumFeatures * 4 + 12);
    double b = 0.5 * (double)free_b / per_anchor;
    b = std::min(b, (double)kMaxBatchPairs / (1.25 * ppa));
    b = std::max(b, (double)(1u << 20));
    return (uint32_t)std::min<double>(b, std::max<uint32_t>(count, 2));
}

int correct_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res, bool copy) {
    if (!ctx) return CARE_B200_EINVAL;
    if (ctx->n == 0) return fail(ctx, CARE_B200_ESTATE, "no reads uploaded");
    if (!ctx->tables_ready) return fail(ctx, CARE_B200_ESTATE, "no tables uploaded or built");
    if ((uint64_t)first + count > ctx->n) return fail(ctx, CARE_B200_EINVAL, "anchor range beyond the read storage");
    if (ctx->opt.paired_end && ((first | count) & 1)) return fail(ctx, CARE_B200_EINVAL, "paired-end ranges must be pair aligned");
    if (ctx->opt.correction_type == 1 && !ctx->mlp_set) return fail(ctx, CARE_B200_ESTATE, "correction_type 1 needs care_b200_set_mlp");
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    if (ctx->sigs_maps != ctx->num_maps)
        if (int rc = compute_signatures(ctx, ctx->num_maps)) return rc;
    ctx->r_fx.clear(); ctx->r_fread.clear(); ctx->r_fmeta.clear(); ctx->r_flogit.clear();
    uint32_t B = ctx->opt.batch_size > 0 ? (uint32_t)ctx->opt.batch_size : auto_batch(ctx, count);
    if (ctx->opt.paired_end) B &= ~1u;
    if (B == 0) B = 2;
    ctx->last_ms = 0.f;
    ctx->stage_ms[0] = ctx->stage_ms[1] = ctx->stage_ms[2] = ctx->stage_ms[3] = 0.f;
    ctx->r_ncand = 0;
    ctx->r_pairs = 0;
    ctx->r_words = 0;
    ctx->r_elems = 0;
    ctx->r_rb_elems = 0;
    ctx->r_rb_anchors = 0;
    ctx->r_batches = 0;
    ctx->r_launches = 0;
    ctx->r_spilled = 0;
    ctx->r_run_words = 0;
    ctx->r_valid = false;
    const int L = ctx->max_len;
    if (copy) {
        CK(ctx->r_status.ensure(std::max<size_t>(count, 1)), "alloc results");
        CK(ctx->r_nedits.ensure((size_t)std::max<size_t>(count, 1) * 4), "alloc results");
        CK(ctx->r_seq.ensure((size_t)std::max<size_t>(count, 1) * L), "alloc results");
    }
    std::vector<uint64_t> corr_counts;
    uint64_t corr_total = 0;
    for (uint32_t b = 0; b < count; b += B) {
        const uint32_t cnt = std::min(B, count - b);
        const uint64_t before = ctx->r_ncand;
        const int rc = run_batch(ctx, first + b, cnt, true);
        if (rc < 0) return rc;
        ctx->r_batches++;
        const uint64_t nc = ctx->r_ncand - before;
        if (copy) {
            CK(cudaMemcpyAsync(ctx->r_status.as<uint8_t>() + b, ctx->d_st.p, cnt, cudaMemcpyDeviceToHost, ctx->stream), "results");
            CK(cudaMemcpyAsync(ctx->r_nedits.as<int32_t>() + b, ctx->d_ned.p, (size_t)cnt * 4, cudaMemcpyDeviceToHost, ctx->stream), "results");
            CK(cudaMemcpyAsync(ctx->r_seq.as<char>() + (size_t)b * L, ctx->d_oseq.p, (size_t)cnt * L, cudaMemcpyDeviceToHost, ctx->stream), "results");
            if (nc) {
                const uint64_t need = corr_total + nc;
                // grow the pinned candidate arrays, keeping earlier batches
                auto grow = [&](HBuf& hb, size_t elem) -> cudaError_t {
                    if (hb.bytes >= need * elem) return cudaSuccess;
                    HBuf nb;
                    const cudaError_t e = nb.ensure(std::max<size_t>(need * elem * 3 / 2, 64));
                    if (e != cudaSuccess) return e;
                    if (hb.p && corr_total) std::memcpy(nb.p, hb.p, corr_total * elem);
                    std::swap(hb.p, nb.p); std::swap(hb.bytes, nb.bytes);
                    return cudaSuccess;
                };
                CK(cudaStreamSynchronize(ctx->stream), "results");
                CK(grow(ctx->r_cid, 4), "alloc"); CK(grow(ctx->r_canc, 4), "alloc"); CK(grow(ctx->r_cshift, 4), "alloc");
                CK(grow(ctx->r_cue, 1), "alloc"); CK(grow(ctx->r_cseq, (size_t)L), "alloc");
                CK(cudaMemcpyAsync(ctx->r_cid.as<uint32_t>() + corr_total, ctx->d_cid.p, nc * 4, cudaMemcpyDeviceToHost, ctx->stream), "results");
                CK(cudaMemcpyAsync(ctx->r_canc.as<uint32_t>() + corr_total, ctx->d_canc.p, nc * 4, cudaMemcpyDeviceToHost, ctx->stream), "results");
                CK(cudaMemcpyAsync(ctx->r_cshift.as<int32_t>() + corr_total, ctx->d_cshift.p, nc * 4, cudaMemcpyDeviceToHost, ctx->stream), "results");
                CK(cudaMemcpyAsync(ctx->r_cue.as<uint8_t>() + corr_total, ctx->d_cue.p, nc, cudaMemcpyDeviceToHost, ctx->stream), "results");
                CK(cudaMemcpyAsync(ctx->r_cseq.as<char>() + corr_total * L, ctx->d_cseq.p, nc * L, cudaMemcpyDeviceToHost, ctx->stream), "results");
            }
            CK(cudaStreamSynchronize(ctx->stream), "results");
        }
        corr_total += nc;
    }
    ctx->r_ncand = corr_total;
    if (count) ctx->pairs_per_anchor = std::max(8.0, (double)ctx->r_pairs / count);
    ctx->r_first = first;
    ctx->r_count = count;
    ctx->r_valid = copy;
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->first_anchor = first;
        res->num_anchors = count;
        res->max_length = L;
        if (copy) {
            res->anchor_status = ctx->r_status.as<uint8_t>();
            res->anchor_num_edits = ctx->r_nedits.as<int32_t>();
            res->anchor_sequences = ctx->r_seq.as<char>();
            res->num_candidates = corr_total;
            res->cand_read_ids = ctx->r_cid.as<uint32_t>();
            res->cand_anchor_ids = ctx->r_canc.as<uint32_t>();
            res->cand_shifts = ctx->r_cshift.as<int32_t>();
            res->cand_use_edits = ctx->r_cue.as<uint8_t>();
            res->cand_sequences = ctx->r_cseq.as<char>();
        }
    }
    return CARE_B200_OK;
}

}  // namespace

extern "C" {

static int care_b200_correct_range_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_correct_range(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res) {
    try {
        return care_b200_correct_range_impl(ctx, first, count, res);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_correct_range: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_correct_range_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res) {
    return correct_impl(ctx, first, count, res, true);
}

static int care_b200_correct_range_device_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_correct_range_device(care_b200_ctx* ctx, uint32_t first, uint32_t count) {
    try {
        return care_b200_correct_range_device_impl(ctx, first, count);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_correct_range_device: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_correct_range_device_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count) {
    return correct_impl(ctx, first, count, nullptr, false);
}

int care_b200_count_word_compares(care_b200_ctx* ctx, int on) {
    if (!ctx || (unsigned)on > 1) return CARE_B200_EINVAL;
    ctx->count_words = on != 0;
    return CARE_B200_OK;
}

int care_b200_default_tuning(care_b200_tuning* t) {
    if (!t) return CARE_B200_EINVAL;
    *t = kDefaultTuning;
    return CARE_B200_OK;
}

int care_b200_set_tuning(care_b200_ctx* ctx, const care_b200_tuning* t) {
    if (!ctx || !t) return CARE_B200_EINVAL;
    if ((t->msa_warps != 4 && t->msa_warps != 8) || (t->align_block != 128 && t->align_block != 256) ||
        (unsigned)t->msa_order > 1 || (unsigned)t->msa_queue > 1 || (unsigned)t->pair_order > 1 ||
        (unsigned)t->graph > 1 || (unsigned)t->pair_mirror > 1 || t->cand_set_log2 < 6 || t->cand_set_log2 > 14 ||
        (unsigned)t->align_warp > 1 || (unsigned)t->align_classes > 1)
        return fail(ctx, CARE_B200_EINVAL, "invalid tuning");
    ctx->tune = *t;
    return CARE_B200_OK;
}

int care_b200_get_tuning(const care_b200_ctx* ctx, care_b200_tuning* t) {
    if (!ctx || !t) return CARE_B200_EINVAL;
    *t = ctx->tune;
    return CARE_B200_OK;
}

static int care_b200_set_mlp_impl(care_b200_ctx* ctx, const float* params);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_set_mlp(care_b200_ctx* ctx, const float* params) {
    try {
        return care_b200_set_mlp_impl(ctx, params);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_set_mlp: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_set_mlp_impl(care_b200_ctx* ctx, const float* params) {
    if (!ctx || !params) return CARE_B200_EINVAL;
    for (int i = 0; i < kMlpFloats; i++)
        if (!std::isfinite(params[i])) return fail(ctx, CARE_B200_EINVAL, "non-finite network parameter");
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    CK(ctx->d_mlp.ensure(kMlpFloats * 4), "alloc network");
    CK(cudaMemcpy(ctx->d_mlp.p, params, kMlpFloats * 4, cudaMemcpyHostToDevice), "upload network");
    ctx->mlp_set = true;
    return CARE_B200_OK;
}

static int care_b200_collect_features_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res,
                               care_b200_features* feats);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_collect_features(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res,
                               care_b200_features* feats) {
    try {
        return care_b200_collect_features_impl(ctx, first, count, res, feats);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_collect_features: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_collect_features_impl(care_b200_ctx* ctx, uint32_t first, uint32_t count, care_b200_results* res,
                               care_b200_features* feats) {
    if (!ctx || !feats) return CARE_B200_EINVAL;
    ctx->collect = true;
    const int rc = correct_impl(ctx, first, count, res, true);
    ctx->collect = false;
    std::memset(feats, 0, sizeof(*feats));
    if (rc) return rc;
    feats->count = ctx->r_fread.size();
    feats->x = ctx->r_fx.data();
    feats->read_ids = ctx->r_fread.data();
    feats->meta = ctx->r_fmeta.data();
    feats->logits = ctx->opt.correction_type == 1 ? ctx->r_flogit.data() : nullptr;
    return CARE_B200_OK;
}

static int care_b200_serialize_results_impl(care_b200_ctx* ctx, const care_b200_results* res, uint8_t* out,
                                size_t capacity, size_t* needed);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_serialize_results(care_b200_ctx* ctx, const care_b200_results* res, uint8_t* out,
                                size_t capacity, size_t* needed) {
    try {
        return care_b200_serialize_results_impl(ctx, res, out, capacity, needed);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_serialize_results: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_serialize_results_impl(care_b200_ctx* ctx, const care_b200_results* res, uint8_t* out,
                                size_t capacity, size_t* needed) {
    if (!ctx || !res || !needed) return CARE_B200_EINVAL;
    size_t pos = 0;
    const int L = res->max_length;
    auto put = [&](const void* p, size_t nb) {
        if (out && pos + nb <= capacity) std::memcpy(out + pos, p, nb);
        pos += nb;
    };
    std::vector<char> dec((size_t)L + 1);
    auto decode = [&](uint32_t id, int len) {
        std::vector<uint32_t> row(ctx->seq_pitch);
        cudaMemcpy(row.data(), ctx->d_seq.as<uint32_t>() + (size_t)id * ctx->seq_pitch, ctx->seq_pitch * 4, cudaMemcpyDeviceToHost);
        for (int p = 0; p < len; p++) dec[p] = "ACGT"[(row[p >> 4] >> (30 - 2 * (p & 15))) & 3u];
    };
    // EncodedTempCorrectedSequence::encodeDataIntoEncodedCorrectedSequence,
    // correctedsequence.hpp:262-336
    auto record = [&](uint32_t id, bool hq, bool useEdits, int type, int shift, const char* seq, int len) {
        std::vector<int> epos;
        std::vector<char> ebase;
        if (useEdits) {
            decode(id, len);
            for (int p = 0; p < len; p++) if (seq[p] != dec[p]) { epos.push_back(p); ebase.push_back(seq[p]); }
        }
        uint32_t nbytes = useEdits ? (uint32_t)(4 + epos.size() * 5) : (uint32_t)(4 + len);
        if (type == 1) nbytes += 4;
        const uint32_t flags = ((uint32_t)hq << 31) | ((uint32_t)useEdits << 30) | ((uint32_t)type << 29) | nbytes;
        put(&id, 4);
        put(&flags, 4);
        if (useEdits) {
            const int ne = (int)epos.size();
            put(&ne, 4);
            for (int p : epos) put(&p, 4);
            for (char c : ebase) put(&c, 1);
        } else {
            put(&len, 4);
            put(seq, (size_t)len);
        }
        if (type == 1) put(&shift, 4);
    };
    for (uint32_t k = 0; k < res->num_anchors; k++) {
        const uint8_t st = res->anchor_status[k];
        if (!(st & 1)) continue;
        const bool hq = st & 2, ue = st & 4;
        if (hq && ue && res->anchor_num_edits[k] == 0) continue;   // correct_cpu.cpp:263-264
        const uint32_t id = res->first_anchor + k;
        record(id, hq, ue, 0, 0, res->anchor_sequences + (size_t)k * L, ctx->h_len[id]);
    }
    for (uint64_t i = 0; i < res->num_candidates; i++) {
        const uint32_t id = res->cand_read_ids[i];
        record(id, false, res->cand_use_edits[i], 1, res->cand_shifts[i], res->cand_sequences + i * L, ctx->h_len[id]);
    }
    *needed = pos;
    if (out && pos > capacity) return fail(ctx, CARE_B200_EINVAL, "serialization buffer too small");
    return CARE_B200_OK;
}

static int care_b200_load_reads_from_files_impl(care_b200_ctx* ctx, const char* const* files, int num_files);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_load_reads_from_files(care_b200_ctx* ctx, const char* const* files, int num_files) {
    try {
        return care_b200_load_reads_from_files_impl(ctx, files, num_files);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_load_reads_from_files: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_load_reads_from_files_impl(care_b200_ctx* ctx, const char* const* files, int num_files) {
    if (!ctx || !files || num_files < 1 || num_files > 2) return CARE_B200_EINVAL;
    std::vector<std::string> fs;
    for (int i = 0; i < num_files; i++) fs.emplace_back(files[i]);
    const std::string e = load_reads(fs, ctx->opt.paired_end, ctx->opt.use_quality, ctx->opt.quality_bits, ctx->reads);
    if (!e.empty()) return fail(ctx, CARE_B200_EIO, e);
    HostReads& h = ctx->reads;
    if (h.n == 0) return fail(ctx, CARE_B200_EINVAL, "no reads in input");
    ctx->have_records = true;
    return care_b200_upload_reads(ctx, h.seq.data(), h.seq_pitch, h.len.data(),
                                  h.has_quality ? h.qual.data() : nullptr, h.qual_pitch,
                                  h.ambiguous_ids.data(), h.ambiguous_ids.size(), h.n);
}

static int care_b200_load_reads_from_files_device_impl(care_b200_ctx* ctx, const char* const* files, int num_files);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_load_reads_from_files_device(care_b200_ctx* ctx, const char* const* files, int num_files) {
    try {
        return care_b200_load_reads_from_files_device_impl(ctx, files, num_files);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_load_reads_from_files_device: ") + e.what())
                   : CARE_B200_ENOMEM;
    }
}

static int care_b200_load_reads_from_files_device_impl(care_b200_ctx* ctx, const char* const* files, int num_files) {
    if (!ctx || !files || num_files < 1 || num_files > 2) return CARE_B200_EINVAL;
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    // the files one after the other in pinned memory, each ending with a line end
    size_t sizes[2] = {0, 0}, begin[2] = {0, 0}, total = 0;
    std::FILE* fp[2] = {nullptr, nullptr};
    auto close_all = [&]() { for (auto& f : fp) if (f) { std::fclose(f); f = nullptr; } };
    for (int f = 0; f < num_files; f++) {
        fp[f] = std::fopen(files[f], "rb");
        if (!fp[f]) { close_all(); return fail(ctx, CARE_B200_EIO, std::string("cannot read input file ") + files[f]); }
        std::fseek(fp[f], 0, SEEK_END);
        const long sz = std::ftell(fp[f]);
        std::fseek(fp[f], 0, SEEK_SET);
        sizes[f] = sz > 0 ? (size_t)sz : 0;
        begin[f] = total;
        total += sizes[f] + 1;
    }
    if (ctx->h_text.ensure(total) != cudaSuccess) { close_all(); return fail(ctx, CARE_B200_ENOMEM, "pinned input buffer"); }
    char* text = ctx->h_text.as<char>();
    size_t used = 0;
    for (int f = 0; f < num_files; f++) {
        begin[f] = used;
        if (sizes[f] && std::fread(text + used, 1, sizes[f], fp[f]) != sizes[f]) {
            close_all();
            return fail(ctx, CARE_B200_EIO, std::string("cannot read input file ") + files[f]);
        }
        used += sizes[f];
        if (sizes[f] == 0 || text[used - 1] != '\n') text[used++] = '\n';
    }
    close_all();
    DeviceParsed dp;
    const std::string e = parse_on_device(text, used, begin, num_files, ctx->opt.paired_end != 0, ctx->opt.use_quality != 0,
                                          ctx->opt.quality_bits, kMaxLen, ctx->stream, dp);
    if (!e.empty()) {
        dp.release();
        if (e == "irregular")
            return fail(ctx, CARE_B200_EINVAL, "records not in strict 4-line FASTQ / 2-line FASTA layout "
                                               "(care_b200_load_reads_from_files reads them)");
        return fail(ctx, e.rfind("reads longer", 0) == 0 ? CARE_B200_ELIMIT : CARE_B200_EIO, e);
    }
    if (ctx->opt.paired_end && (dp.n % 2)) {
        dp.release();
        return fail(ctx, CARE_B200_EINVAL, "paired-end storage needs an even number of reads");
    }
    // the device arrays become the read storage
    ctx->d_seq.adopt(dp.seq, (size_t)dp.n * dp.seq_pitch * 4);
    ctx->d_len.adopt(dp.len, (size_t)dp.n * 4);
    ctx->d_ambig.adopt(dp.ambig, dp.n);
    if (dp.has_quality) ctx->d_qual.adopt(dp.qual, (size_t)dp.n * dp.qual_pitch * 4);
    ctx->n = dp.n;
    ctx->max_len = dp.max_len;
    ctx->seq_pitch = dp.seq_pitch;
    ctx->has_qual = dp.has_quality;
    ctx->qual_pitch = dp.has_quality ? dp.qual_pitch : 0;
    ctx->h_len = dp.h_len;
    ctx->h_ambig = dp.h_ambig;
    HostReads& h = ctx->reads;
    h = HostReads{};
    h.n = dp.n;
    h.min_len = dp.min_len;
    h.max_len = dp.max_len;
    h.seq_pitch = dp.seq_pitch;
    h.qual_pitch = dp.qual_pitch;
    h.quality_bits = ctx->opt.quality_bits;
    h.has_quality = dp.has_quality;
    h.fasta = dp.fasta;
    h.seq = std::move(dp.h_seq);
    h.len = std::move(dp.h_len);
    h.ambig = std::move(dp.h_ambig);
    for (uint32_t i = 0; i < h.n; i++) if (h.ambig[i]) h.ambiguous_ids.push_back(i);
    h.raw = text;
    h.rec_h = std::move(dp.rec_h);
    h.rec_hl = std::move(dp.rec_hl);
    h.rec_s = std::move(dp.rec_s);
    h.rec_q = std::move(dp.rec_q);
    ctx->have_records = true;
    ctx->sigs_maps = 0;
    if (int rc = compute_signatures(ctx, ctx->num_maps ? ctx->num_maps : ctx->opt.num_maps)) return rc;
    CK(cudaStreamSynchronize(ctx->stream), "signatures");
    if (ctx->tables_ready && ctx->t_keys.size() && h.n != ctx->tables_reads) ctx->tables_ready = false;
    ctx->r_valid = false;
    return CARE_B200_OK;
}

static int care_b200_load_preprocessed_reads_impl(care_b200_ctx* ctx, const char* path);

// The file formats are parsed with std::vector: an allocation failure is
// returned as an error code, nothing is thrown across the C ABI.
int care_b200_load_preprocessed_reads(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    try {
        return care_b200_load_preprocessed_reads_impl(ctx, path);
    } catch (const std::exception& e) {
        return fail(ctx, CARE_B200_ENOMEM, std::string("load_preprocessed_reads: ") + e.what());
    }
}

static int care_b200_load_preprocessed_reads_impl(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    ReadStorageFile f;
    const std::string e = read_storage_file(path, f);
    if (!e.empty()) return fail(ctx, CARE_B200_EIO, e);
    const bool useq = ctx->opt.use_quality != 0;
    if (useq && !f.has_quality)
        return fail(ctx, CARE_B200_EINVAL, "quality scores expected in the read-storage file, but none are present");
    if (useq && f.quality_bits != ctx->opt.quality_bits)
        return fail(ctx, CARE_B200_EINVAL, "the read-storage file uses " + std::to_string(f.quality_bits) +
                                               " bits per quality score, the options " +
                                               std::to_string(ctx->opt.quality_bits));
    // output records of an earlier care_b200_load_reads_from_files stay in
    // use for the same reads (care-cpu writes its output from the input files)
    ctx->have_records = ctx->have_records && ctx->reads.n == f.n;
    return care_b200_upload_reads(ctx, f.seq.data(), f.seq_pitch, f.len.data(),
                                  useq ? f.qual.data() : nullptr, f.qual_pitch, f.ambiguous_ids.data(),
                                  f.ambiguous_ids.size(), (uint32_t)f.n);
}

static int care_b200_save_preprocessed_reads_impl(care_b200_ctx* ctx, const char* path);

// The file formats are parsed with std::vector: an allocation failure is
// returned as an error code, nothing is thrown across the C ABI.
int care_b200_save_preprocessed_reads(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    try {
        return care_b200_save_preprocessed_reads_impl(ctx, path);
    } catch (const std::exception& e) {
        return fail(ctx, CARE_B200_ENOMEM, std::string("save_preprocessed_reads: ") + e.what());
    }
}

static int care_b200_save_preprocessed_reads_impl(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    if (ctx->n == 0) return fail(ctx, CARE_B200_ESTATE, "no reads uploaded");
    CK(cudaSetDevice(ctx->opt.device), "cudaSetDevice");
    ReadStorageFile f;
    f.n = ctx->n;
    f.has_quality = ctx->has_qual;
    f.quality_bits = ctx->opt.quality_bits;
    f.seq_pitch = (uint64_t)ctx->seq_pitch;
    f.qual_pitch = ctx->has_qual ? (uint64_t)ctx->qual_pitch : 0;
    f.seq.resize(f.n * f.seq_pitch);
    f.len.resize(f.n);
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    CK(cudaMemcpy(f.seq.data(), ctx->d_seq.p, f.seq.size() * 4, cudaMemcpyDeviceToHost), "download sequences");
    CK(cudaMemcpy(f.len.data(), ctx->d_len.p, f.len.size() * 4, cudaMemcpyDeviceToHost), "download lengths");
    if (f.has_quality) {
        f.qual.resize(f.n * f.qual_pitch);
        CK(cudaMemcpy(f.qual.data(), ctx->d_qual.p, f.qual.size() * 4, cudaMemcpyDeviceToHost), "download qualities");
    }
    f.min_len = *std::min_element(f.len.begin(), f.len.end());
    f.max_len = *std::max_element(f.len.begin(), f.len.end());
    for (uint32_t i = 0; i < ctx->n; ++i)
        if (ctx->h_ambig[i]) f.ambiguous_ids.push_back(i);
    const std::string e = write_storage_file(path, f);
    if (!e.empty()) return fail(ctx, CARE_B200_EIO, e);
    return CARE_B200_OK;
}

static int care_b200_load_hashtables_impl(care_b200_ctx* ctx, const char* path);

// The file formats are parsed with std::vector: an allocation failure is
// returned as an error code, nothing is thrown across the C ABI.
int care_b200_load_hashtables(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    try {
        return care_b200_load_hashtables_impl(ctx, path);
    } catch (const std::exception& e) {
        return fail(ctx, CARE_B200_ENOMEM, std::string("load_hashtables: ") + e.what());
    }
}

static int care_b200_load_hashtables_impl(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    if (ctx->n == 0) return fail(ctx, CARE_B200_ESTATE, "no reads uploaded");
    MinhashTablesFile t;
    const std::string e = read_tables_file(path, t, ctx->opt.num_maps);
    if (!e.empty()) return fail(ctx, CARE_B200_EIO, e);
    for (const auto& v : t.values)
        for (uint32_t id : v)
            if (id >= ctx->n) return fail(ctx, CARE_B200_EINVAL, "table holds a read id beyond the read storage");
    // as the reference's loader: k and the per-map result threshold of the file
    if (t.k != ctx->opt.kmerlength) {
        ctx->opt.kmerlength = t.k;
        ctx->sigs_maps = 0;                 // signatures of the storage are hashed again with this k
    }
    ctx->threshold = t.threshold;
    const int maps = (int)t.keys.size();
    std::vector<const uint64_t*> k(maps);
    std::vector<const uint32_t*> o(maps), v(maps);
    std::vector<size_t> nk(maps);
    for (int m = 0; m < maps; ++m) {
        k[m] = t.keys[m].data();
        o[m] = t.offsets[m].data();
        v[m] = t.values[m].data();
        nk[m] = t.keys[m].size();
    }
    return care_b200_upload_tables(ctx, maps, k.data(), o.data(), v.data(), nk.data());
}

static int care_b200_save_hashtables_impl(care_b200_ctx* ctx, const char* path);

// The file formats are parsed with std::vector: an allocation failure is
// returned as an error code, nothing is thrown across the C ABI.
int care_b200_save_hashtables(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    try {
        return care_b200_save_hashtables_impl(ctx, path);
    } catch (const std::exception& e) {
        return fail(ctx, CARE_B200_ENOMEM, std::string("save_hashtables: ") + e.what());
    }
}

static int care_b200_save_hashtables_impl(care_b200_ctx* ctx, const char* path) {
    if (!ctx || !path) return CARE_B200_EINVAL;
    if (!ctx->tables_ready) return fail(ctx, CARE_B200_ESTATE, "no tables uploaded or built");
    MinhashTablesFile t;
    t.k = ctx->opt.kmerlength;
    t.threshold = ctx->threshold;
    t.load = 0.8f;                          // the reference's default hashtable load factor
    for (int m = 0; m < ctx->num_maps; ++m) {
        const uint64_t* keys = nullptr;
        const uint32_t* offs = nullptr;
        const uint32_t* vals = nullptr;
        size_t nk = 0;
        if (int rc = care_b200_get_table(ctx, m, &keys, &offs, &vals, &nk)) return rc;
        t.keys.emplace_back(keys, keys + nk);
        t.offsets.emplace_back(offs, offs + nk + 1);
        t.values.emplace_back(vals, vals + (nk ? offs[nk] : 0));
    }
    const std::string e = write_tables_file(path, t);
    if (!e.empty()) return fail(ctx, CARE_B200_EIO, e);
    return CARE_B200_OK;
}

static int care_b200_write_output_impl(care_b200_ctx* ctx, const char* outfile);

// host allocations that fail are returned as CARE_B200_ENOMEM: nothing is
// thrown across the C ABI
int care_b200_write_output(care_b200_ctx* ctx, const char* outfile) {
    try {
        return care_b200_write_output_impl(ctx, outfile);
    } catch (const std::exception& e) {
        return ctx ? fail(ctx, CARE_B200_ENOMEM, std::string("care_b200_write_output: ") + e.what()) : CARE_B200_ENOMEM;
    }
}

static int care_b200_write_output_impl(care_b200_ctx* ctx, const char* outfile) {
    if (!ctx || !outfile) return CARE_B200_EINVAL;
    if (!ctx->have_records) return fail(ctx, CARE_B200_ESTATE, "reads were not loaded from files");
    if (!ctx->r_valid) return fail(ctx, CARE_B200_ESTATE, "no correction results");
    HostCorrections c;
    c.first = ctx->r_first;
    c.count = ctx->r_count;
    c.max_len = ctx->max_len;
    c.status = ctx->r_status.as<uint8_t>();
    c.nedits = ctx->r_nedits.as<int32_t>();
    c.seq = ctx->r_seq.as<char>();
    c.ncand = ctx->r_ncand;
    c.cand_id = ctx->r_cid.as<uint32_t>();
    c.cand_use_edits = ctx->r_cue.as<uint8_t>();
    c.cand_seq = ctx->r_cseq.as<char>();
    const std::string e = write_corrected(ctx->reads, c, ctx->opt.quality_labels, outfile);
    if (!e.empty()) return fail(ctx, CARE_B200_EIO, e);
    return CARE_B200_OK;
}

int care_b200_last_timing(const care_b200_ctx* ctx, float* total_ms, float* stage_ms, int nstages) {
    if (!ctx) return CARE_B200_EINVAL;
    if (total_ms) *total_ms = ctx->last_ms;
    for (int i = 0; i < nstages && i < 4 && stage_ms; i++) stage_ms[i] = ctx->stage_ms[i];
    if (stage_ms && nstages > 4) {
        float ms = 0.f;
        for (int k = 0; k + 1 < ctx->sig_used; k += 2) {
            float part = 0.f;
            if (cudaEventSynchronize(ctx->sig_ev[k + 1]) == cudaSuccess &&
                cudaEventElapsedTime(&part, ctx->sig_ev[k], ctx->sig_ev[k + 1]) == cudaSuccess)
                ms += part;
        }
        stage_ms[4] = ms;
    }
    return CARE_B200_OK;
}

int care_b200_last_stats(const care_b200_ctx* ctx, uint64_t* stats, int nstats) {
    if (!ctx || !stats) return CARE_B200_EINVAL;
    const uint64_t v[11] = {ctx->r_count, ctx->r_pairs, ctx->r_ncand, ctx->r_words, ctx->r_elems, ctx->r_batches,
                            ctx->r_launches, ctx->r_spilled, ctx->r_run_words, ctx->r_rb_elems, ctx->r_rb_anchors};
    for (int i = 0; i < nstats && i < 11; i++) stats[i] = v[i];
    return CARE_B200_OK;
}

uint32_t care_b200_num_reads(const care_b200_ctx* ctx) { return ctx ? ctx->n : 0; }
int care_b200_max_length(const care_b200_ctx* ctx) { return ctx ? ctx->max_len : 0; }
int care_b200_num_maps(const care_b200_ctx* ctx) { return ctx ? ctx->num_maps : 0; }
int care_b200_result_threshold(const care_b200_ctx* ctx) { return ctx ? ctx->threshold : 0; }

}  // extern "C"
