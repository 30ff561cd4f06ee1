// hostio.cpp -- input parsing, read preprocessing and output construction.
#include "hostio.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <thread>

namespace careb200 {

namespace {

struct FileBuf {
    std::vector<char> data;
    size_t pos = 0;
};

bool read_whole(const std::string& path, FileBuf& f) {
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    const long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    f.data.resize(sz > 0 ? (size_t)sz : 0);
    const bool ok = sz <= 0 || std::fread(f.data.data(), 1, (size_t)sz, fp) == (size_t)sz;
    std::fclose(fp);
    f.pos = 0;
    return ok;
}

struct Rec {
    const char* h; size_t hl;
    const char* s; size_t sl;
    const char* q; size_t ql;
    bool fasta;
};

// One record of a 4-line FASTQ or single-line FASTA file, read at `pos`
// (advanced past it) of the n bytes at d.
bool next_record_at(const char* d, size_t n, size_t& pos, Rec& r) {
    while (pos < n && d[pos] != '@' && d[pos] != '>') pos++;
    if (pos >= n) return false;
    r.fasta = d[pos] == '>';
    auto line = [&](size_t p, const char*& b, size_t& l) {
        size_t e = p;
        while (e < n && d[e] != '\n') e++;
        b = d + p;
        l = e - p;
        if (l && b[l - 1] == '\r') l--;
        return e + 1;
    };
    size_t p = line(pos + 1, r.h, r.hl);
    p = line(p, r.s, r.sl);
    if (r.fasta) { r.q = ""; r.ql = 0; pos = p; return true; }
    const char* plus; size_t pl;
    p = line(p, plus, pl);
    p = line(p, r.q, r.ql);
    pos = p;
    return true;
}

// Start of the first record at or after `from`: a line that starts with '>'
// (FASTA), or with '@' and has a '+' line two lines below (FASTQ; a quality
// line that starts with '@' is followed by a header and a sequence line, so it
// never passes). n when there is none.
size_t record_start(const char* d, size_t n, size_t from, bool fasta) {
    auto next_line = [&](size_t p) {
        while (p < n && d[p] != '\n') p++;
        return p < n ? p + 1 : n;
    };
    size_t p = from;
    if (p > 0 && d[p - 1] != '\n') p = next_line(p);
    for (; p < n; p = next_line(p)) {
        if (fasta) { if (d[p] == '>') return p; continue; }
        if (d[p] != '@') continue;
        const size_t l2 = next_line(next_line(p));
        if (l2 < n && d[l2] == '+') return p;
    }
    return n;
}

// All records of a file, as a scan from its first byte finds them. Up to
// `threads` threads scan segments that begin at record starts; the segments
// must chain (each scan ends exactly where the next segment begins), else the
// file is scanned again from the beginning by one thread.
std::vector<Rec> scan_file(const FileBuf& f, unsigned threads) {
    const char* d = f.data.data();
    const size_t n = f.data.size();
    std::vector<Rec> all;
    auto serial = [&]() {
        all.clear();
        size_t pos = 0;
        Rec r;
        while (next_record_at(d, n, pos, r)) all.push_back(r);
    };
    const unsigned T = (unsigned)std::max<size_t>(1, std::min<size_t>(threads, n >> 16));   // >= 64 KB a segment
    size_t first = 0;
    while (first < n && d[first] != '@' && d[first] != '>') first++;
    if (T <= 1 || first >= n) { serial(); return all; }
    const bool fasta = d[first] == '>';
    std::vector<size_t> start(T + 1, n);
    start[0] = first;
    for (unsigned t = 1; t < T; t++) start[t] = std::max(start[t - 1], record_start(d, n, n / T * t, fasta));
    std::vector<std::vector<Rec>> part(T);
    std::vector<size_t> endpos(T, 0);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++) {
        th.emplace_back([&, t] {
            size_t pos = start[t];
            Rec r;
            while (pos < start[t + 1] && next_record_at(d, n, pos, r)) part[t].push_back(r);
            endpos[t] = std::max(pos, start[t]);
        });
    }
    for (auto& x : th) x.join();
    for (unsigned t = 0; t + 1 < T; t++)
        if (endpos[t] != start[t + 1]) { serial(); return all; }
    size_t total = 0;
    for (auto& v : part) total += v.size();
    all.reserve(total);
    for (auto& v : part) all.insert(all.end(), v.begin(), v.end());
    return all;
}

}  // namespace

void encode_2bit(const char* s, int len, uint32_t* out) {
    const int n = (len + 15) / 16;
    for (int i = 0; i < n; i++) {
        uint32_t w = 0;
        const int b = i * 16, e = std::min(len, b + 16);
        for (int p = b; p < e; p++) {
            uint32_t c = 0;
            switch (s[p]) { case 'C': c = 1; break; case 'G': c = 2; break; case 'T': c = 3; break; default: c = 0; }
            w = (w << 2) | c;
        }
        w <<= 2 * (16 - (e - b));
        out[i] = w;
    }
}

int quality_ints(int len, int bits) { return (bits * len + 31) / 32; }

// qualityscorecompression.hpp:90-119 (1/2-bit binning), :284-287 (8-bit copy)
void encode_quality(const char* q, int len, int bits, uint32_t* out) {
    const int n = quality_ints(len, bits);
    if (bits == 8) {
        std::memset(out, 0, (size_t)n * 4);
        std::memcpy(out, q, (size_t)len);
        return;
    }
    static const int b1[2] = {13, 256}, b2[4] = {4, 13, 20, 256};
    const int* bound = bits == 1 ? b1 : b2;
    const int nb = 1 << bits, per = 32 / bits;
    for (int w = 0; w < n; w++) {
        uint32_t d = 0;
        const int pend = std::min(len, (w + 1) * per);
        for (int p = w * per; p < pend; p++) {
            const int Q = (int)(unsigned char)q[p] - 33;
            for (int x = 0; x < nb; x++)
                if (Q <= bound[x]) { d = (d << bits) | (uint32_t)x; break; }
        }
        if (w == n - 1) d <<= ((w + 1) * per - len) * bits;
        out[w] = d;
    }
}

void quality_weights(float* w) {
    for (int i = 0; i < 256; i++) {
        const float p = i < 33 ? 1.0f : std::pow(10.0f, -(i - 33) / 10.0f);
        w[i] = std::max(0.001f, 1.0f - p);
    }
}

std::string load_reads(const std::vector<std::string>& files, bool paired_end, bool use_quality,
                       int quality_bits, HostReads& out) {
    return load_reads_threads(files, paired_end, use_quality, quality_bits, out,
                              std::max(1u, std::thread::hardware_concurrency()));
}

std::string load_reads_threads(const std::vector<std::string>& files, bool paired_end, bool use_quality,
                               int quality_bits, HostReads& out, unsigned threads) {
    if (files.empty() || files.size() > 2) return "expected one or two input files";
    threads = std::max(1u, threads);
    std::vector<FileBuf> in(files.size());
    for (size_t i = 0; i < files.size(); i++)
        if (!read_whole(files[i], in[i])) return "cannot read input file " + files[i];

    out = HostReads{};
    out.quality_bits = quality_bits;
    std::vector<size_t> fileFirst;      // first read of each SE file (rotation restarts)
    fileFirst.push_back(0);
    // records in read order: one file; two SE files one after the other; two
    // PE files alternating (mate 1, mate 2, ...) until either file ends
    std::vector<Rec> recs;
    {
        std::vector<std::vector<Rec>> per(files.size());
        for (size_t i = 0; i < files.size(); i++) per[i] = scan_file(in[i], threads);
        if (files.size() == 1) {
            recs = std::move(per[0]);
        } else if (!paired_end) {
            recs = std::move(per[0]);
            fileFirst.push_back(recs.size());
            recs.insert(recs.end(), per[1].begin(), per[1].end());
        } else {
            for (size_t i = 0;; i++) {
                if (i >= per[0].size()) break;
                recs.push_back(per[0][i]);
                if (i >= per[1].size()) break;
                recs.push_back(per[1][i]);
            }
        }
    }
    const size_t n = recs.size();
    // the records' text, NUL separated: header, sequence, quality
    out.rec_off.resize(n);
    out.len.resize(n);
    size_t tsize = 0;
    for (size_t i = 0; i < n; i++) {
        const Rec& r = recs[i];
        out.fasta |= r.fasta;
        out.rec_off[i] = tsize;
        out.len[i] = (int32_t)r.sl;
        tsize += r.hl + r.sl + r.ql + 3;
    }
    out.text.resize(tsize);
    {
        const unsigned T = (unsigned)std::max<size_t>(1, std::min<size_t>(threads, n / 4096));
        std::vector<std::thread> th;
        for (unsigned t = 0; t < T; t++) {
            th.emplace_back([&, t] {
                for (size_t i = n * t / T; i < n * (t + 1) / T; i++) {
                    const Rec& r = recs[i];
                    char* o = out.text.data() + out.rec_off[i];
                    std::memcpy(o, r.h, r.hl); o += r.hl; *o++ = 0;
                    std::memcpy(o, r.s, r.sl); o += r.sl; *o++ = 0;
                    std::memcpy(o, r.q, r.ql); o += r.ql; *o++ = 0;
                }
            });
        }
        for (auto& x : th) x.join();
    }
    if (n >= 0xFFFFFFFFu) return "too many reads";
    out.n = (uint32_t)n;
    out.has_quality = use_quality && !out.fasta;
    int mn = n ? 1 << 30 : 0, mx = 0;
    for (size_t i = 0; i < n; i++) { mn = std::min(mn, out.len[i]); mx = std::max(mx, out.len[i]); }
    out.min_len = mn;
    out.max_len = mx;
    out.seq_pitch = (mx + 15) / 16;
    out.qual_pitch = quality_ints(mx, quality_bits);
    out.seq.assign(n * (size_t)out.seq_pitch, 0u);
    if (out.has_quality) out.qual.assign(n * (size_t)out.qual_pitch, 0u);
    out.ambig.assign(n, 0);

    // preprocessSequence (chunkedreadstorageconstruction.hpp:67-92): lower case
    // letters are upper-cased; other characters become A,C,G,T in turn, with
    // the turn counter reset at the start of every 65536-read parser batch.
    // batches are independent given their start; process whole batches per thread
    std::vector<std::pair<size_t, size_t>> batches;
    for (size_t fi = 0; fi < fileFirst.size(); fi++) {
        const size_t fb = fileFirst[fi], fe = fi + 1 < fileFirst.size() ? fileFirst[fi + 1] : n;
        for (size_t b = fb; b < fe; b += 65536) batches.push_back({b, std::min(fe, b + 65536)});
    }
    // process each batch sequentially inside (rotation carries within a batch)
    auto batch_work = [&](size_t bi0, size_t bi1) {
        std::vector<char> tmp((size_t)mx + 1);
        for (size_t bi = bi0; bi < bi1; bi++) {
            int Ncount = 0;
            for (size_t i = batches[bi].first; i < batches[bi].second; i++) {
                const char* h = out.text.data() + out.rec_off[i];
                const char* s = h + std::strlen(h) + 1;
                const int L = out.len[i];
                bool und = false;
                for (int p = 0; p < L; p++) {
                    char c = s[p];
                    if (c == 'a') c = 'A'; else if (c == 'c') c = 'C'; else if (c == 'g') c = 'G'; else if (c == 't') c = 'T';
                    else if (!(c == 'A' || c == 'C' || c == 'G' || c == 'T')) {
                        und = true;
                        c = "ACGT"[Ncount];
                        Ncount = (Ncount + 1) % 4;
                    }
                    tmp[p] = c;
                }
                out.ambig[i] = und;
                encode_2bit(tmp.data(), L, out.seq.data() + i * out.seq_pitch);
                if (out.has_quality)
                    encode_quality(s + L + 1, L, quality_bits, out.qual.data() + i * out.qual_pitch);
            }
        }
    };
    const size_t nb = batches.size();
    const unsigned nt = std::max(1u, std::min<unsigned>(threads, (unsigned)nb));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) th.emplace_back(batch_work, nb * t / nt, nb * (t + 1) / nt);
    for (auto& x : th) x.join();
    for (size_t i = 0; i < n; i++) if (out.ambig[i]) out.ambiguous_ids.push_back((uint32_t)i);
    return "";
}

std::string write_corrected(const HostReads& reads, const HostCorrections& c, bool quality_labels,
                            const std::string& path) {
    std::FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return "cannot open output file " + path;
    const int dp = c.max_len;
    const uint32_t n = reads.n;
    // candidate corrections grouped by read id, in stored order within a read
    // (a stable counting sort); read i's are order[cstart[i] .. cstart[i+1])
    std::vector<uint64_t> cstart((size_t)n + 1, 0), order;
    for (uint64_t k = 0; k < c.ncand; k++)
        if (c.cand_id[k] < n) cstart[c.cand_id[k] + 1]++;
    for (uint32_t i = 0; i < n; i++) cstart[i + 1] += cstart[i];
    order.resize(cstart[n]);
    {
        std::vector<uint64_t> fill(cstart.begin(), cstart.end() - 1);
        for (uint64_t k = 0; k < c.ncand; k++)
            if (c.cand_id[k] < n) order[fill[c.cand_id[k]]++] = k;
    }
    // The reference's merge (correctionresultoutput.cpp:30-440) combines --
    // and labels -- only reads up to the last read id with a stored result;
    // later reads are copied unchanged. Stored results: anchor results that
    // pass the save filter, candidate results for reads that are not HQ
    // anchors (corrector.hpp:1682-1684 drops those once the flag is set).
    int64_t last = -1;
    for (uint32_t k = 0; k < c.count; k++) {
        const uint8_t st = c.status[k];
        if ((st & 1) && !((st & 2) && (st & 4) && c.nedits[k] == 0)) last = std::max<int64_t>(last, c.first + k);
    }
    for (uint64_t k = 0; k < c.ncand; k++) {
        const uint32_t id = c.cand_id[k];
        const bool hqAnchor = id >= c.first && id < c.first + c.count && (c.status[id - c.first] & 3) == 3;
        if (!hqAnchor) last = std::max<int64_t>(last, id);
    }

    // the output records of reads [b, e) appended to buf
    auto format = [&](uint32_t b, uint32_t e, std::string& buf) {
        std::vector<char> dec((size_t)reads.max_len + 1), m0((size_t)reads.max_len + 1),
            m1((size_t)reads.max_len + 1), outseq((size_t)reads.max_len + 1);
        auto decode = [&](uint32_t id, int L) {
            const uint32_t* row = reads.seq.data() + (size_t)id * reads.seq_pitch;
            for (int p = 0; p < L; p++) dec[p] = "ACGT"[(row[p >> 4] >> (30 - 2 * (p & 15))) & 3u];
        };
        // the sequence the combiner writes for one result: edits applied to
        // the input read, or the stored full sequence
        auto materialize = [&](const char* orig, const char* seq, int L, bool useEdits, char* o) {
            if (useEdits) {
                std::memcpy(o, orig, (size_t)L);
                for (int i = 0; i < L; i++) if (seq[i] != dec[i]) o[i] = seq[i];
            } else std::memcpy(o, seq, (size_t)L);
        };
        for (uint32_t i = b; i < e; i++) {
            const int L = reads.len[i];
            const char *h, *s, *q;
            size_t hl, ql;
            if (reads.raw) {
                h = reads.raw + reads.rec_h[i];
                hl = reads.rec_hl[i];
                s = reads.raw + reads.rec_s[i];
                q = reads.raw + reads.rec_q[i];
                ql = reads.fasta ? 0 : (size_t)L;
            } else {
                h = reads.text.data() + reads.rec_off[i];
                hl = std::strlen(h);
                s = h + hl + 1;
                q = s + std::strlen(s) + 1;
                ql = std::strlen(q);
            }
            std::memcpy(outseq.data(), s, (size_t)L);
            const uint64_t cb = cstart[i], ce = cstart[i + 1];
            const uint64_t ncand = ce - cb;
            int label = 0;
            bool corrected = false;
            if (i >= c.first && i < c.first + c.count) {
                const uint32_t k = i - c.first;
                const uint8_t st = c.status[k];
                const bool isCorr = st & 1, hq = st & 2, useEdits = st & 4;
                // correct_cpu.cpp:263-264 save filter: HQ edit lists with no
                // edit are not stored
                const bool stored = isCorr && !(hq && useEdits && c.nedits[k] == 0);
                if (stored) {
                    const char* aseq = c.seq + (size_t)k * dp;
                    decode(i, L);
                    if (hq) {
                        materialize(s, aseq, L, useEdits, outseq.data());
                        corrected = true; label = 3;
                    } else if (1 + ncand >= 3) {
                        materialize(s, aseq, L, useEdits, m0.data());
                        bool same = true;
                        for (uint64_t x = cb; x < ce && same; x++) {
                            const uint64_t idx = order[x];
                            materialize(s, c.cand_seq + idx * dp, L, c.cand_use_edits[idx], m1.data());
                            if (std::memcmp(m0.data(), m1.data(), (size_t)L) != 0) same = false;
                        }
                        if (same) { std::memcpy(outseq.data(), m0.data(), (size_t)L); corrected = true; label = 2; }
                    } else {
                        materialize(s, aseq, L, useEdits, outseq.data());
                        corrected = true; label = 1;
                    }
                }
            }
            buf.push_back(reads.fasta ? '>' : '@');
            buf.append(h, hl);
            if (quality_labels && (int64_t)i <= last) { buf.append(" care:q="); buf.push_back((char)('0' + (corrected ? label : 0))); }
            buf.push_back('\n');
            buf.append(outseq.data(), (size_t)L);
            buf.push_back('\n');
            if (!reads.fasta) { buf.append("+\n"); buf.append(q, ql); buf.push_back('\n'); }
        }
    };
    // blocks of reads formatted by threads, written in read order
    const unsigned T = std::max(1u, std::thread::hardware_concurrency());
    const uint32_t block = 1u << 20;
    std::vector<std::string> bufs(T);
    bool ok = true;
    for (uint32_t b0 = 0; b0 < n && ok; b0 += block) {
        const uint32_t b1 = (uint32_t)std::min<uint64_t>((uint64_t)b0 + block, n);
        const unsigned use = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(T, (b1 - b0) / 1024));
        std::vector<std::thread> th;
        for (unsigned t = 0; t < use; t++) {
            th.emplace_back([&, t] {
                bufs[t].clear();
                format(b0 + (uint32_t)((uint64_t)(b1 - b0) * t / use), b0 + (uint32_t)((uint64_t)(b1 - b0) * (t + 1) / use),
                       bufs[t]);
            });
        }
        for (auto& x : th) x.join();
        for (unsigned t = 0; t < use && ok; t++)
            ok = std::fwrite(bufs[t].data(), 1, bufs[t].size(), fp) == bufs[t].size();
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? "" : "write error on " + path;
}

}  // namespace careb200
