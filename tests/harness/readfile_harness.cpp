// Host harness for the read-storage file (care_b200/csrc/readfile.cpp) and
// this library's FASTQ preprocessing (care_b200/csrc/hostio.cpp), for the
// CPU tests: C entry points over plain arrays.
#include <cstring>
#include <string>

#include "../../care_b200/csrc/hostio.hpp"
#include "../../care_b200/csrc/readfile.hpp"

using namespace careb200;

namespace {
void set_err(const std::string& e, char* err, int n) {
    if (err && n > 0) { std::strncpy(err, e.c_str(), n - 1); err[n - 1] = 0; }
}
}  // namespace

extern "C" {

// the file's storage; info = n, min, max, has quality, quality bits, seq pitch, qual pitch, ambiguous count
void* rf_load(const char* path, unsigned long long* info, char* err, int errlen) {
    auto* f = new ReadStorageFile;
    const std::string e = read_storage_file(path, *f);
    if (!e.empty()) { set_err(e, err, errlen); delete f; return nullptr; }
    const unsigned long long v[8] = {f->n, (unsigned long long)f->min_len, (unsigned long long)f->max_len,
                                     f->has_quality, (unsigned long long)f->quality_bits, f->seq_pitch,
                                     f->qual_pitch, f->ambiguous_ids.size()};
    std::memcpy(info, v, sizeof(v));
    return f;
}

void rf_arrays(void* h, uint32_t* seq, int32_t* len, uint32_t* qual, uint32_t* ambig) {
    const auto* f = static_cast<const ReadStorageFile*>(h);
    std::memcpy(seq, f->seq.data(), f->seq.size() * 4);
    std::memcpy(len, f->len.data(), f->len.size() * 4);
    if (!f->qual.empty()) std::memcpy(qual, f->qual.data(), f->qual.size() * 4);
    if (!f->ambiguous_ids.empty()) std::memcpy(ambig, f->ambiguous_ids.data(), f->ambiguous_ids.size() * 4);
}

void rf_free(void* h) { delete static_cast<ReadStorageFile*>(h); }

int rf_write(const char* path, unsigned long long n, int minl, int maxl, int hasq, int qbits,
             unsigned long long sp, unsigned long long qp, const uint32_t* seq, const int32_t* len,
             const uint32_t* qual, const uint32_t* ambig, unsigned long long na, char* err, int errlen) {
    ReadStorageFile f;
    f.n = n; f.min_len = minl; f.max_len = maxl; f.has_quality = hasq != 0; f.quality_bits = qbits;
    f.seq_pitch = sp; f.qual_pitch = qp;
    f.seq.assign(seq, seq + n * sp);
    f.len.assign(len, len + n);
    if (hasq) f.qual.assign(qual, qual + n * qp);
    f.ambiguous_ids.assign(ambig, ambig + na);
    const std::string e = write_storage_file(path, f);
    set_err(e, err, errlen);
    return e.empty() ? 0 : -1;
}

// this library's STEP1 preprocessing of one FASTQ file; same info layout
void* rf_parse(const char* path, int paired_end, int quality_bits, unsigned long long* info, char* err, int errlen) {
    auto* h = new HostReads;
    const std::string e = load_reads({std::string(path)}, paired_end != 0, true, quality_bits, *h);
    if (!e.empty()) { set_err(e, err, errlen); delete h; return nullptr; }
    const unsigned long long v[8] = {h->n, (unsigned long long)h->min_len, (unsigned long long)h->max_len,
                                     h->has_quality, (unsigned long long)h->quality_bits,
                                     (unsigned long long)h->seq_pitch, (unsigned long long)h->qual_pitch,
                                     h->ambiguous_ids.size()};
    std::memcpy(info, v, sizeof(v));
    return h;
}

void rf_parse_arrays(void* p, uint32_t* seq, int32_t* len, uint32_t* qual, uint32_t* ambig) {
    const auto* h = static_cast<const HostReads*>(p);
    std::memcpy(seq, h->seq.data(), h->seq.size() * 4);
    std::memcpy(len, h->len.data(), h->len.size() * 4);
    if (!h->qual.empty()) std::memcpy(qual, h->qual.data(), h->qual.size() * 4);
    if (!h->ambiguous_ids.empty()) std::memcpy(ambig, h->ambiguous_ids.data(), h->ambiguous_ids.size() * 4);
}

void rf_parse_free(void* p) { delete static_cast<HostReads*>(p); }

// FNV-1a digest of everything this library's preprocessing produces for one
// or two files with `threads` threads: read count, record text and offsets,
// lengths, 2-bit rows, quality rows, ambiguous ids
int rf_parse_digest(const char* f0, const char* f1, int paired_end, int quality_bits, unsigned threads,
                    unsigned long long* digest, unsigned long long* nreads, char* err, int errlen) {
    HostReads h;
    std::vector<std::string> files{f0};
    if (f1) files.push_back(f1);
    const std::string e = load_reads_threads(files, paired_end != 0, true, quality_bits, h, threads);
    if (!e.empty()) { set_err(e, err, errlen); return -1; }
    unsigned long long x = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t bytes) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < bytes; i++) { x ^= c[i]; x *= 1099511628211ull; }
    };
    mix(&h.n, sizeof(h.n));
    mix(h.text.data(), h.text.size());
    mix(h.rec_off.data(), h.rec_off.size() * sizeof(size_t));
    mix(h.len.data(), h.len.size() * 4);
    mix(h.seq.data(), h.seq.size() * 4);
    mix(h.qual.data(), h.qual.size() * 4);
    mix(h.ambiguous_ids.data(), h.ambiguous_ids.size() * 4);
    *digest = x;
    *nreads = h.n;
    return 0;
}

// minhash-table file: info = k, threshold, maps, load factor bits
void* rt_load(const char* path, int max_maps, unsigned long long* info, char* err, int errlen) {
    auto* t = new MinhashTablesFile;
    const std::string e = read_tables_file(path, *t, max_maps);
    if (!e.empty()) { set_err(e, err, errlen); delete t; return nullptr; }
    uint32_t lb;
    std::memcpy(&lb, &t->load, 4);
    const unsigned long long v[4] = {(unsigned long long)t->k, (unsigned long long)t->threshold, t->keys.size(), lb};
    std::memcpy(info, v, sizeof(v));
    return t;
}

void rt_map_size(void* h, int m, unsigned long long* nkeys, unsigned long long* nvalues) {
    const auto* t = static_cast<const MinhashTablesFile*>(h);
    *nkeys = t->keys[m].size();
    *nvalues = t->values[m].size();
}

void rt_map(void* h, int m, uint64_t* keys, uint32_t* offsets, uint32_t* values) {
    const auto* t = static_cast<const MinhashTablesFile*>(h);
    std::memcpy(keys, t->keys[m].data(), t->keys[m].size() * 8);
    std::memcpy(offsets, t->offsets[m].data(), t->offsets[m].size() * 4);
    std::memcpy(values, t->values[m].data(), t->values[m].size() * 4);
}

int rt_write(void* h, const char* path, char* err, int errlen) {
    const std::string e = write_tables_file(path, *static_cast<const MinhashTablesFile*>(h));
    set_err(e, err, errlen);
    return e.empty() ? 0 : -1;
}

void rt_free(void* h) { delete static_cast<MinhashTablesFile*>(h); }

}  // extern "C"
