// parse.cu -- STEP1 on the device: the input files' bytes are copied to the
// device once, the line ends found by a device-wide scan, the records laid
// out from them, and the reads encoded by one warp each. The result is the
// storage the host parse (hostio.cpp) builds from the same bytes:
//   record layout      hostio.cpp next_record_at (4-line FASTQ, 2-line FASTA)
//   preprocessing      chunkedreadstorageconstruction.hpp:67-92 (upper case;
//                      other characters become A, C, G, T in turn, the turn
//                      counter restarting every 65,536-read parser batch,
//                      :106 and :259)
//   2-bit sequences    sequencehelpers.hpp encodeSequence2Bit (MSB first)
//   quality encoding   qualityscorecompression.hpp:90-119 (1/2-bit bins) and
//                      :284-287 (8-bit copy)
// The turn counter is the one sequential dependence: it becomes an exclusive
// scan of each read's count of ambiguous characters within its batch, then a
// warp scan over the read's 16-character words.
#include "parse.hpp"

#include <algorithm>
#include <cstring>

namespace careb200 {

namespace {

constexpr size_t kTile = 1u << 16;            // bytes per line-end tile
constexpr int kTileThreads = 256;             // 256 bytes per thread
constexpr uint32_t kBatchReads = 65536;       // the reference parser's batch of reads
constexpr int kIrregular = 1, kTooLong = 2;

__device__ __forceinline__ int newlines_in(uint32_t w) {
    return __popc(__vcmpeq4(w, 0x0A0A0A0Au)) >> 3;
}

// line ends per tile
__global__ void __launch_bounds__(kTileThreads)
k_nl_count(const uint4* __restrict__ text, unsigned* __restrict__ tile_cnt) {
    const uint4* p = text + (size_t)blockIdx.x * (kTile / 16) + threadIdx.x * 16;
    int c = 0;
#pragma unroll 4
    for (int i = 0; i < 16; ++i) {
        const uint4 v = p[i];
        c += newlines_in(v.x) + newlines_in(v.y) + newlines_in(v.z) + newlines_in(v.w);
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ int s[kTileThreads / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kTileThreads / 32; ++w) t += s[w];
        tile_cnt[blockIdx.x] = (unsigned)t;
    }
}

// exclusive scan of n values in one CTA (1024 threads), the total at out[n]
template <class T>
__global__ void __launch_bounds__(1024) k_scan_one(const T* __restrict__ in, unsigned long long* __restrict__ out,
                                                    size_t n) {
    __shared__ unsigned long long s[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (size_t b = 0; b < n; b += 1024) {
        const size_t i = b + threadIdx.x;
        const unsigned long long v = i < n ? (unsigned long long)in[i] : 0ull;
        unsigned long long x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) s[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long z = s[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, z, d);
                if (lane >= d) z += y;
            }
            s[lane] = z;                       // inclusive over warps
        }
        __syncthreads();
        const unsigned long long pre = carry + (warp ? s[warp - 1] : 0ull) + x - v;
        if (i < n) out[i] = pre;
        __syncthreads();
        if (threadIdx.x == 1023) carry = pre + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// positions of the line ends, in order
__global__ void __launch_bounds__(kTileThreads)
k_nl_write(const unsigned char* __restrict__ text, const unsigned long long* __restrict__ tile_off,
           unsigned long long* __restrict__ nl) {
    const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * 256;
    const uint4* p = reinterpret_cast<const uint4*>(text + base);
    int c = 0;
#pragma unroll 4
    for (int i = 0; i < 16; ++i) {
        const uint4 v = p[i];
        c += newlines_in(v.x) + newlines_in(v.y) + newlines_in(v.z) + newlines_in(v.w);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    __shared__ int s[kTileThreads / 32];
    if (lane == 31) s[warp] = x;
    __syncthreads();
    int pre = x - c;
    for (int w = 0; w < warp; ++w) pre += s[w];
    unsigned long long o = tile_off[blockIdx.x] + (unsigned long long)pre;
    for (int i = 0; i < 256 && c; ++i) {
        if (text[base + i] == '\n') { nl[o++] = base + i; --c; }
    }
}

// first line of each file: line ends before its first byte
__global__ void k_file_lines(const unsigned long long* __restrict__ nl, unsigned long long nlines,
                             const unsigned long long* __restrict__ fbeg, int nfiles,
                             unsigned long long* __restrict__ first_line) {
    const int f = threadIdx.x;
    if (f > nfiles) return;
    const unsigned long long x = fbeg[f];
    unsigned long long lo = 0, hi = nlines;
    while (lo < hi) {
        const unsigned long long mid = (lo + hi) >> 1;
        if (nl[mid] < x) lo = mid + 1; else hi = mid;
    }
    first_line[f] = lo;
}

struct FileRecs {
    unsigned long long line0;      // first line of the file
    unsigned long long count;      // records of the file
    unsigned long long out0;       // combined index of record 0 (SE), or file index (PE)
};

// one thread per record of one file: its lines, the layout checks, and its
// offsets. fasta: records of 2 lines ('>' header), else 4 ('@', sequence,
// '+', quality of the sequence's length). pe: record i of file f goes to
// 2i + f when kept (the host's alternating order), else to out0 + i.
__global__ void k_records(const unsigned char* __restrict__ text, const unsigned long long* __restrict__ nl,
                          FileRecs fr, int file, bool pe, unsigned long long keep, bool fasta,
                          unsigned long long* __restrict__ rec_h, uint32_t* __restrict__ rec_hl,
                          unsigned long long* __restrict__ rec_s, unsigned long long* __restrict__ rec_q,
                          int32_t* __restrict__ len, int max_len_limit, int* __restrict__ flags,
                          int* __restrict__ minmax) {
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= keep) return;
    const int per = fasta ? 2 : 4;
    const unsigned long long g = fr.line0 + i * per;
    auto start = [&](unsigned long long l) { return l == 0 ? 0ull : nl[l - 1] + 1; };
    auto stop = [&](unsigned long long l) {
        const unsigned long long s0 = start(l), e = nl[l];
        return (e > s0 && text[e - 1] == '\r') ? e - 1 : e;
    };
    const unsigned long long hs = start(g), he = stop(g);
    const unsigned long long ss = start(g + 1), se = stop(g + 1);
    bool ok = hs < nl[g] && text[hs] == (fasta ? '>' : '@');
    unsigned long long qs = 0;
    if (!fasta) {
        const unsigned long long ps = start(g + 2);
        qs = start(g + 3);
        const unsigned long long qe = stop(g + 3);
        ok = ok && ps < nl[g + 2] && text[ps] == '+' && qe - qs == se - ss;
    }
    if (!ok) { atomicOr(flags, kIrregular); return; }
    const unsigned long long L = se - ss;
    if (L > (unsigned long long)max_len_limit) { atomicOr(flags, kTooLong); return; }
    const unsigned long long r = pe ? 2 * i + file : fr.out0 + i;
    rec_h[r] = hs + 1;
    rec_hl[r] = (uint32_t)(he - hs - 1);
    rec_s[r] = ss;
    rec_q[r] = qs;
    len[r] = (int32_t)L;
    atomicMin(&minmax[0], (int)L);
    atomicMax(&minmax[1], (int)L);
}

__device__ __forceinline__ int base_code(unsigned char c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return -1;                    // ambiguous: takes the turn counter's base
    }
}

// ambiguous characters per read (warp per read)
__global__ void k_ambig_count(const unsigned char* __restrict__ text, const unsigned long long* __restrict__ rec_s,
                              const int32_t* __restrict__ len, uint32_t n, uint32_t* __restrict__ cnt) {
    const uint32_t r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (r >= n) return;
    const int lane = threadIdx.x & 31;
    const unsigned char* s = text + rec_s[r];
    const int L = len[r];
    int c = 0;
    for (int p = lane; p < L; p += 32) c += base_code(s[p]) < 0;
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) cnt[r] = (uint32_t)c;
}

// per parser batch (one CTA each): the turn counter at each read's start,
// an exclusive scan of the ambiguous counts within the batch, modulo 4
__global__ void __launch_bounds__(1024) k_batch_turns(const uint32_t* __restrict__ cnt,
                                                      const uint32_t* __restrict__ bstart, uint8_t* __restrict__ turn) {
    const uint32_t b0 = bstart[blockIdx.x], b1 = bstart[blockIdx.x + 1];
    __shared__ uint32_t s[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b = b0; b < b1; b += 1024) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < b1 ? cnt[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) s[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t z = s[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
                if (lane >= d) z += y;
            }
            s[lane] = z;
        }
        __syncthreads();
        const uint32_t pre = carry + (warp ? s[warp - 1] : 0u) + x - v;
        if (i < b1) turn[i] = (uint8_t)(pre & 3u);
        __syncthreads();
        if (threadIdx.x == 1023) carry = pre + v;
        __syncthreads();
    }
}

// encoding, a warp per read: lane w packs sequence word w (16 bases), the
// turn counter carried over the words by a warp scan; quality words after
__global__ void k_encode(const unsigned char* __restrict__ text, const unsigned long long* __restrict__ rec_s,
                         const unsigned long long* __restrict__ rec_q, const int32_t* __restrict__ len,
                         const uint8_t* __restrict__ turn, const uint32_t* __restrict__ cnt, uint32_t n, int sp,
                         int qp, int qbits, uint32_t* __restrict__ seq, uint32_t* __restrict__ qual,
                         uint8_t* __restrict__ ambig) {
    const uint32_t r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (r >= n) return;
    const int lane = threadIdx.x & 31;
    const int L = len[r];
    const unsigned char* s = text + rec_s[r];
    const int nw = (L + 15) >> 4;             // <= 16 words (reads of at most 256 bases)
    int amb = 0;
    if (lane < nw) {
        const int e = min(L, 16 * lane + 16);
        for (int p = 16 * lane; p < e; ++p) amb += base_code(s[p]) < 0;
    }
    int x = amb;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane < nw) {
        int t = (int)((turn[r] + (uint32_t)(x - amb)) & 3u);
        const int b = 16 * lane, e = min(L, b + 16);
        uint32_t w = 0;
        for (int p = b; p < e; ++p) {
            int c = base_code(s[p]);
            if (c < 0) { c = t; t = (t + 1) & 3; }
            w = (w << 2) | (uint32_t)c;
        }
        w <<= 2 * (16 - (e - b));
        seq[(size_t)r * sp + lane] = w;
    }
    if (lane == 0) ambig[r] = cnt[r] != 0;
    if (qual) {
        const unsigned char* q = text + rec_q[r];
        const int nq = (qbits * L + 31) / 32;
        for (int wq = lane; wq < nq; wq += 32) {
            uint32_t d = 0;
            if (qbits == 8) {
                for (int k = 0; k < 4; ++k) {
                    const int p = 4 * wq + k;
                    if (p < L) d |= (uint32_t)q[p] << (8 * k);
                }
            } else {
                const int per = 32 / qbits;
                const int b = wq * per, e = min(L, b + per);
                for (int p = b; p < e; ++p) {
                    const int Q = (int)q[p] - 33;
                    const uint32_t bin = qbits == 1 ? (Q <= 13 ? 0u : 1u)
                                                    : (Q <= 4 ? 0u : Q <= 13 ? 1u : Q <= 20 ? 2u : 3u);
                    d = (d << qbits) | bin;
                }
                d <<= (uint32_t)((b + per - e) * qbits);
            }
            qual[(size_t)r * qp + wq] = d;
        }
    }
}

struct Dev {
    void* p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, n ? n : 16); }
    void* take() { void* q = p; p = nullptr; return q; }
};

}  // namespace

void DeviceParsed::release() {
    if (seq) cudaFree(seq);
    if (qual) cudaFree(qual);
    if (len) cudaFree(len);
    if (ambig) cudaFree(ambig);
    seq = qual = nullptr;
    len = nullptr;
    ambig = nullptr;
}

#define PK(call, what) do { const cudaError_t e_ = (call); if (e_ != cudaSuccess) return std::string(what) + ": " + cudaGetErrorString(e_); } while (0)

std::string parse_on_device(const char* text, size_t text_bytes, const size_t* file_begin, int num_files,
                            bool paired_end, bool use_quality, int quality_bits, int max_len_limit,
                            cudaStream_t st, DeviceParsed& out) {
    out = DeviceParsed{};
    if (num_files < 1 || num_files > 2 || text_bytes == 0) return "expected one or two input files";
    const bool fasta = text[file_begin[0]] == '>';
    for (int f = 0; f < num_files; f++) {
        const size_t e = f + 1 < num_files ? file_begin[f + 1] : text_bytes;
        if (file_begin[f] >= e || text[file_begin[f]] != (fasta ? '>' : '@') || text[e - 1] != '\n')
            return "irregular";
    }
    // the bytes, zero padded to whole tiles
    const size_t ntiles = (text_bytes + kTile - 1) / kTile;
    Dev d_text, d_tcnt, d_toff;
    PK(d_text.alloc(ntiles * kTile), "alloc text");
    PK(cudaMemsetAsync(d_text.as<char>() + text_bytes, 0, ntiles * kTile - text_bytes, st), "memset");
    PK(cudaMemcpyAsync(d_text.p, text, text_bytes, cudaMemcpyHostToDevice, st), "copy text");
    PK(d_tcnt.alloc(ntiles * 4), "alloc");
    PK(d_toff.alloc((ntiles + 1) * 8), "alloc");
    k_nl_count<<<(unsigned)ntiles, kTileThreads, 0, st>>>(d_text.as<uint4>(), d_tcnt.as<unsigned>());
    k_scan_one<unsigned><<<1, 1024, 0, st>>>(d_tcnt.as<unsigned>(), d_toff.as<unsigned long long>(), ntiles);
    unsigned long long nlines = 0;
    PK(cudaMemcpyAsync(&nlines, d_toff.as<unsigned long long>() + ntiles, 8, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaStreamSynchronize(st), "line ends");
    Dev d_nl, d_fb, d_fl;
    PK(d_nl.alloc(nlines * 8), "alloc line ends");
    k_nl_write<<<(unsigned)ntiles, kTileThreads, 0, st>>>(d_text.as<unsigned char>(), d_toff.as<unsigned long long>(),
                                                          d_nl.as<unsigned long long>());
    unsigned long long fb[3] = {file_begin[0], num_files > 1 ? file_begin[1] : text_bytes, text_bytes};
    fb[num_files] = text_bytes;
    PK(d_fb.alloc(sizeof(fb)), "alloc");
    PK(d_fl.alloc(sizeof(fb)), "alloc");
    PK(cudaMemcpyAsync(d_fb.p, fb, sizeof(fb), cudaMemcpyHostToDevice, st), "copy");
    k_file_lines<<<1, 32, 0, st>>>(d_nl.as<unsigned long long>(), nlines, d_fb.as<unsigned long long>(), num_files,
                                   d_fl.as<unsigned long long>());
    unsigned long long fl[3] = {0, 0, 0};
    PK(cudaMemcpyAsync(fl, d_fl.p, sizeof(fl), cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaStreamSynchronize(st), "line ends");
    PK(cudaGetLastError(), "line-end kernels");

    // records per file, the combined order of the host parse
    const int per = fasta ? 2 : 4;
    unsigned long long cnt[2] = {0, 0};
    for (int f = 0; f < num_files; f++) {
        const unsigned long long lines = fl[f + 1] - fl[f];
        if (lines % per) return "irregular";
        cnt[f] = lines / per;
    }
    unsigned long long n = cnt[0], keep[2] = {cnt[0], 0};
    const bool pe2 = num_files == 2 && paired_end;
    if (num_files == 2) {
        if (pe2) {          // mate 1, mate 2, ... until either file ends (host loop order)
            const unsigned long long m = std::min(cnt[0], cnt[1]);
            keep[0] = cnt[0] > cnt[1] ? m + 1 : m;
            keep[1] = m;
            n = keep[0] + keep[1];
        } else {
            keep[1] = cnt[1];
            n = cnt[0] + cnt[1];
        }
    }
    if (n == 0) return "no reads in input";
    if (n >= 0xFFFFFFFFull) return "too many reads";
    Dev d_rh, d_rhl, d_rs, d_rq, d_len, d_flags, d_mm;
    PK(d_rh.alloc(n * 8), "alloc");
    PK(d_rhl.alloc(n * 4), "alloc");
    PK(d_rs.alloc(n * 8), "alloc");
    PK(d_rq.alloc(n * 8), "alloc");
    PK(d_len.alloc(n * 4), "alloc");
    PK(d_flags.alloc(16), "alloc");
    PK(d_mm.alloc(8), "alloc");
    const int mm0[2] = {0x7fffffff, 0};
    PK(cudaMemsetAsync(d_flags.p, 0, 16, st), "memset");
    PK(cudaMemcpyAsync(d_mm.p, mm0, 8, cudaMemcpyHostToDevice, st), "copy");
    for (int f = 0; f < num_files; f++) {
        if (!keep[f]) continue;
        const FileRecs fr{fl[f], cnt[f], f == 0 ? 0ull : cnt[0]};
        k_records<<<(unsigned)((keep[f] + 255) / 256), 256, 0, st>>>(
            d_text.as<unsigned char>(), d_nl.as<unsigned long long>(), fr, f, pe2, keep[f], fasta,
            d_rh.as<unsigned long long>(), d_rhl.as<uint32_t>(), d_rs.as<unsigned long long>(),
            d_rq.as<unsigned long long>(), d_len.as<int32_t>(), max_len_limit, d_flags.as<int>(), d_mm.as<int>());
    }
    int flags = 0, mm[2];
    PK(cudaMemcpyAsync(&flags, d_flags.p, 4, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(mm, d_mm.p, 8, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaStreamSynchronize(st), "records");
    PK(cudaGetLastError(), "record kernel");
    if (flags & kIrregular) return "irregular";
    if (flags & kTooLong) return "reads longer than 256 bases are not supported";

    // ambiguous counts, the turn counter per parser batch, encoding
    const uint32_t N = (uint32_t)n;
    std::vector<uint32_t> bst;
    const uint32_t second = (num_files == 2 && !paired_end) ? (uint32_t)cnt[0] : N;   // SE files restart it
    for (uint32_t b = 0; b < second; b += kBatchReads) bst.push_back(b);
    for (uint32_t b = second; b < N; b += kBatchReads) bst.push_back(b);
    bst.push_back(N);
    Dev d_cnt, d_bst, d_turn;
    PK(d_cnt.alloc((size_t)N * 4), "alloc");
    PK(d_bst.alloc(bst.size() * 4), "alloc");
    PK(d_turn.alloc(N), "alloc");
    PK(cudaMemcpyAsync(d_bst.p, bst.data(), bst.size() * 4, cudaMemcpyHostToDevice, st), "copy");
    const unsigned wblocks = (N + 7) / 8;      // 8 warps per CTA
    k_ambig_count<<<wblocks, 256, 0, st>>>(d_text.as<unsigned char>(), d_rs.as<unsigned long long>(),
                                           d_len.as<int32_t>(), N, d_cnt.as<uint32_t>());
    k_batch_turns<<<(unsigned)(bst.size() - 1), 1024, 0, st>>>(d_cnt.as<uint32_t>(), d_bst.as<uint32_t>(),
                                                               d_turn.as<uint8_t>());
    out.n = N;
    out.min_len = mm[0];
    out.max_len = mm[1];
    out.fasta = fasta;
    out.has_quality = use_quality && !fasta;
    out.seq_pitch = (out.max_len + 15) / 16;
    out.qual_pitch = (quality_bits * out.max_len + 31) / 32;
    if (out.seq_pitch == 0) out.seq_pitch = 1;
    Dev d_seq, d_qual, d_amb;
    PK(d_seq.alloc((size_t)N * out.seq_pitch * 4), "alloc reads");
    PK(cudaMemsetAsync(d_seq.p, 0, (size_t)N * out.seq_pitch * 4, st), "memset");
    if (out.has_quality) {
        PK(d_qual.alloc((size_t)N * out.qual_pitch * 4), "alloc qualities");
        PK(cudaMemsetAsync(d_qual.p, 0, (size_t)N * out.qual_pitch * 4, st), "memset");
    }
    PK(d_amb.alloc(N), "alloc");
    k_encode<<<wblocks, 256, 0, st>>>(d_text.as<unsigned char>(), d_rs.as<unsigned long long>(),
                                      d_rq.as<unsigned long long>(), d_len.as<int32_t>(), d_turn.as<uint8_t>(),
                                      d_cnt.as<uint32_t>(), N, out.seq_pitch, out.qual_pitch, quality_bits,
                                      d_seq.as<uint32_t>(), out.has_quality ? d_qual.as<uint32_t>() : nullptr,
                                      d_amb.as<uint8_t>());
    PK(cudaGetLastError(), "encode kernels");
    out.h_len.resize(N);
    out.h_ambig.resize(N);
    out.h_seq.resize((size_t)N * out.seq_pitch);
    out.rec_h.resize(N);
    out.rec_hl.resize(N);
    out.rec_s.resize(N);
    out.rec_q.resize(N);
    PK(cudaMemcpyAsync(out.h_len.data(), d_len.p, (size_t)N * 4, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(out.h_ambig.data(), d_amb.p, N, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(out.h_seq.data(), d_seq.p, out.h_seq.size() * 4, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(out.rec_h.data(), d_rh.p, (size_t)N * 8, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(out.rec_hl.data(), d_rhl.p, (size_t)N * 4, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(out.rec_s.data(), d_rs.p, (size_t)N * 8, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaMemcpyAsync(out.rec_q.data(), d_rq.p, (size_t)N * 8, cudaMemcpyDeviceToHost, st), "copy");
    PK(cudaStreamSynchronize(st), "encode");
    out.seq = static_cast<uint32_t*>(d_seq.take());
    out.qual = out.has_quality ? static_cast<uint32_t*>(d_qual.take()) : nullptr;
    out.len = static_cast<int32_t*>(d_len.take());
    out.ambig = static_cast<uint8_t*>(d_amb.take());
    return "";
}

}  // namespace careb200
