/*
 * care_oracle.c -- CPU restatement of CARE's per-anchor correction path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product). Sequential
 * plain C; each function cites the reference (yanlifeng/CARE) file:line it
 * restates. Pinned against the reference's own care-cpu built from source
 * (oracle/_ref/care-cpu): see tests/test_oracle_pin.py.
 *
 * Floating point: every float expression is written so that it evaluates in
 * the same order as the reference, and the file is compiled with
 * -ffp-contract=off (no fused multiply-add), matching the reference build in
 * oracle/Makefile.
 */
#define _GNU_SOURCE
#include "care_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define MAXK 32

static void* xmalloc(size_t n) {
    void* p = malloc(n ? n : 1);
    if (!p) { fprintf(stderr, "care-oracle: out of memory\n"); exit(2); }
    return p;
}
static void* xcalloc(size_t n, size_t s) {
    void* p = calloc(n ? n : 1, s ? s : 1);
    if (!p) { fprintf(stderr, "care-oracle: out of memory\n"); exit(2); }
    return p;
}

/* include/options.hpp:37-98 */
void co_default_opts(co_opts* o) {
    memset(o, 0, sizeof(*o));
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
    o->threads = 1;
    o->clf_min_coverage = 3;
}

/* ------------------------------------------------------------------ */
/* 2-bit sequences: include/sequencehelpers.hpp                          */
/* ------------------------------------------------------------------ */

static int ints2bit(int len) { return (len + 15) / 16; }       /* :146-148 */
static int ints2bithilo(int len) { return 2 * ((len + 31) / 32); }

static uint32_t enc_base(char c) {                               /* :135-143 */
    switch (c) { case 'A': return 0; case 'C': return 1; case 'G': return 2; case 'T': return 3; }
    return 0;
}
static char dec_base(uint32_t b) { return "ACGT"[b & 3]; }       /* :124-132 */

/* encodeSequence2Bit, sequencehelpers.hpp:152-187 */
void co_encode_2bit(const char* s, int len, uint32_t* out) {
    const int n = ints2bit(len);
    for (int i = 0; i < n; i++) out[i] = 0;
    for (int p = 0; p < len; p++) out[p / 16] = (out[p / 16] << 2) | enc_base(s[p]);
    const int left = 2 * (n * 16 - len);
    if (left > 0) out[n - 1] <<= left;
}

/* decode2BitSequence, sequencehelpers.hpp:196-225 */
void co_decode_2bit(const uint32_t* enc, int len, char* out) {
    for (int i = 0; i < len; i++) out[i] = dec_base(enc[i / 16] >> (30 - 2 * (i % 16)));
}

/* EncodedReverseComplement2Bit<unsigned>::compute_, sequencehelpers.hpp:18-26 */
static uint32_t rc_word(uint32_t n) {
    n = ((n >> 2) & 0x33333333u) | ((n & 0x33333333u) << 2);
    n = ((n >> 4) & 0x0F0F0F0Fu) | ((n & 0x0F0F0F0Fu) << 4);
    n = ((n >> 8) & 0x00FF00FFu) | ((n & 0x00FF00FFu) << 8);
    n = ((n >> 16) & 0x0000FFFFu) | ((n & 0x0000FFFFu) << 16);
    return 0xFFFFFFFFu - n;
}

/* reverseComplementSequence2Bit / ...Inplace2Bit, sequencehelpers.hpp:267-324 */
void co_revcomp_2bit(const uint32_t* in, int len, uint32_t* out) {
    const int n = ints2bit(len);
    const int unused = n * 16 - len;
    for (int i = 0; i < n; i++) out[i] = in[i];
    for (int i = 0; i < n / 2; i++) {
        const uint32_t front = rc_word(out[i]);
        const uint32_t back = rc_word(out[n - 1 - i]);
        out[i] = back;
        out[n - 1 - i] = front;
    }
    if (n % 2 == 1) out[n / 2] = rc_word(out[n / 2]);
    if (unused > 0) {
        for (int i = 0; i < n - 1; i++)
            out[i] = (out[i] << (2 * unused)) | (out[i + 1] >> (2 * (16 - unused)));
        out[n - 1] <<= (2 * unused);
    }
}

/* extractEvenBits + convert2BitTo2BitHiLo, sequencehelpers.hpp:645-697 */
static uint32_t even_bits(uint32_t x) {
    x = x & 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    x = (x | (x >> 8)) & 0x0000FFFFu;
    return x;
}
void co_to_hilo(const uint32_t* in, int len, uint32_t* out) {
    const int nin = ints2bit(len), nout = ints2bithilo(len);
    uint32_t* hi = out;
    uint32_t* lo = out + nout / 2;
    for (int i = 0; i < nout; i++) out[i] = 0;
    for (int i = 0; i < nin; i++) {
        const uint32_t e = even_bits(in[i]), o = even_bits(in[i] >> 1);
        if (i % 2 == 0) { hi[i / 2] = o << 16; lo[i / 2] = e << 16; }
        else { hi[i / 2] |= o; lo[i / 2] |= e; }
    }
}

static void revcomp_decoded(const char* s, int len, char* out) { /* sequencehelpers.hpp:45-56 */
    for (int i = 0; i < len; i++) {
        char c = s[i], r = c;
        switch (c) { case 'A': r = 'T'; break; case 'C': r = 'G'; break;
                     case 'G': r = 'C'; break; case 'T': r = 'A'; break; }
        out[len - 1 - i] = r;
    }
}

/* ------------------------------------------------------------------ */
/* Minhash: include/cpusequencehasher.hpp:88-125,                       */
/* sequencehelpers.hpp:844-926, hpc_helpers hashers.cuh:85-139          */
/* (MurmurHash3's 64-bit finalizer, a published algorithm)              */
/* ------------------------------------------------------------------ */

uint64_t co_murmur64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

static uint64_t rc_kmer64(uint64_t n) { /* EncodedReverseComplement2Bit<u64>, :27-34 */
    n = ((n >> 2) & 0x3333333333333333ull) | ((n & 0x3333333333333333ull) << 2);
    n = ((n >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((n & 0x0F0F0F0F0F0F0F0Full) << 4);
    n = ((n >> 8) & 0x00FF00FF00FF00FFull) | ((n & 0x00FF00FF00FF00FFull) << 8);
    n = ((n >> 16) & 0x0000FFFF0000FFFFull) | ((n & 0x0000FFFF0000FFFFull) << 16);
    n = ((n >> 32) & 0x00000000FFFFFFFFull) | ((n & 0x00000000FFFFFFFFull) << 32);
    return ~0ull - n;
}

static uint64_t kmer_at(const uint32_t* s, int k, int pos) { /* :699-722 */
    const uint64_t mask = ~0ull >> ((MAXK - k) * 2);
    uint64_t kmer = 0;
    while (k > 0) {
        const int ii = pos / 16;
        const uint64_t d = s[ii];
        int need = 16 - (pos % 16);
        if (k < need) need = k;
        const int sh = 2 * (16 - need - (pos % 16));
        kmer = (kmer << (2 * need)) | (d >> sh);
        k -= need;
        pos += need;
    }
    return kmer & mask;
}

/* CPUSequenceHasher::hashInto with firstHashFunc = 0 (cpusequencehasher.hpp:88-125)
 * over forEachEncodedCanonicalKmerFromEncodedSequence (sequencehelpers.hpp:844-926). */
void co_signature(const uint32_t* seq, int len, int k, int num_maps, uint64_t* out) {
    const uint64_t mask = ~0ull >> ((MAXK - k) * 2);
    for (int h = 0; h < num_maps; h++) out[h] = ~0ull;
    if (len >= k) {
        const int rcshift = (MAXK - k) * 2;
        uint64_t kmer = kmer_at(seq, k, 0) >> 2;
        uint64_t rc = rc_kmer64(kmer);
        for (int next = k - 1; next < len; next++) {
            const uint64_t b = (uint64_t)(seq[next / 16] >> (30 - 2 * (next % 16)));
            kmer = ((kmer << 2) | b) & mask;
            rc = (rc >> 2) | (((~b) & 3ull) << 62);
            const uint64_t fw = kmer, rv = rc >> rcshift;
            const uint64_t canon = fw < rv ? fw : rv;
            for (int h = 0; h < num_maps; h++) {
                const uint64_t v = co_murmur64(canon + (uint64_t)h);
                if (v < out[h]) out[h] = v;
            }
        }
    }
    for (int h = 0; h < num_maps; h++) out[h] &= mask;
}

/* calculateResultsPerMapThreshold, minhasherlimit.hpp:9-15; the coverage is
 * passed as an int (cpuminhasherconstruction.cpp:186-191). */
int co_threshold(float coverage) {
    const int cov = (int)coverage;
    int r = (int)(cov * 2.5f);
    if (r > 65535) r = 65535;
    if (r < 10) r = 10;
    return r;
}

/* ------------------------------------------------------------------ */
/* Quality scores: include/qualityscorecompression.hpp:25-145,          */
/* include/qualityscoreweights.hpp:12-44                                */
/* ------------------------------------------------------------------ */

static int qual_ints(int len, int bits) { return (bits * len + 31) / 32; }

void co_encode_quality(const char* q, int len, int bits, uint32_t* out) {
    const int n = qual_ints(len, bits);
    if (bits == 8) {                                   /* :284-287, memcpy */
        memset(out, 0, (size_t)n * 4);
        memcpy(out, q, (size_t)len);
        return;
    }
    static const int bound1[2] = {13, 256}, bound2[4] = {4, 13, 20, 256};
    const int* bound = bits == 1 ? bound1 : bound2;
    const int nb = 1 << bits, per = 32 / bits;
    for (int w = 0; w < n; w++) {                      /* :95-119 */
        uint32_t d = 0;
        int pend = (w + 1) * per;
        if (pend > len) pend = len;
        for (int p = w * per; p < pend; p++) {
            const int Q = (int)(unsigned char)q[p] - 33;
            for (int x = 0; x < nb; x++)
                if (Q <= bound[x]) { d = (d << bits) | (uint32_t)x; break; }
        }
        if (w == n - 1) d <<= ((w + 1) * per - len) * bits;
        out[w] = d;
    }
}

void co_decode_quality(const uint32_t* enc, int len, int bits, char* out) {
    if (bits == 8) { memcpy(out, enc, (size_t)len); return; }   /* :289-291 */
    static const char bin1[2] = {'(', '5'}, bin2[4] = {'$', '(', '1', '9'};
    const char* bin = bits == 1 ? bin1 : bin2;
    const int per = 32 / bits;
    for (int p = 0; p < len; p++) {                    /* :121-145 */
        const int w = p / per, pos = p - w * per;
        const uint32_t b = (enc[w] >> ((32 - bits) - pos * bits)) & ((1u << bits) - 1);
        out[p] = bin[b];
    }
}

/* QualityScoreConversion constructor, qualityscoreweights.hpp:16-31 */
void co_quality_weights(float* w) {
    for (int i = 0; i < 256; i++) {
        const float p = i < 33 ? 1.0f : powf(10.0f, -(i - 33) / 10.0f);
        const float v = 1.0f - p;
        w[i] = 0.001f > v ? 0.001f : v;
    }
}

/* ------------------------------------------------------------------ */
/* Read storage construction: chunkedreadstorageconstruction.hpp        */
/* ------------------------------------------------------------------ */

typedef struct { char* buf; size_t len, cap; } sbuf;
static void sb_put(sbuf* b, const char* s, size_t n) {
    if (b->len + n + 1 > b->cap) {
        size_t c = b->cap ? b->cap : 1 << 20;
        while (c < b->len + n + 1) c *= 2;
        b->buf = realloc(b->buf, c);
        if (!b->buf) { fprintf(stderr, "care-oracle: out of memory\n"); exit(2); }
        b->cap = c;
    }
    memcpy(b->buf + b->len, s, n);
    b->len += n;
    b->buf[b->len] = 0;
}

typedef struct {
    char* data; size_t size, pos;
} infile;

static int load_file(const char* path, infile* f) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return -1;
    fseek(fp, 0, SEEK_END);
    long sz = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    f->data = xmalloc((size_t)sz + 1);
    if (sz > 0 && fread(f->data, 1, (size_t)sz, fp) != (size_t)sz) { fclose(fp); return -1; }
    f->data[sz] = 0;
    f->size = (size_t)sz;
    f->pos = 0;
    fclose(fp);
    return 0;
}

/* Reads one record: header (after '@'/'>'), sequence, quality (empty for
 * FASTA). 4-line FASTQ and single-line FASTA records. Returns 0 at EOF. */
static int next_record(infile* f, const char** h, size_t* hl, const char** s, size_t* sl,
                       const char** q, size_t* ql, int* fasta) {
    while (f->pos < f->size && f->data[f->pos] != '@' && f->data[f->pos] != '>') f->pos++;
    if (f->pos >= f->size) return 0;
    *fasta = f->data[f->pos] == '>';
    size_t p = f->pos + 1, e;
    e = p; while (e < f->size && f->data[e] != '\n') e++;
    *h = f->data + p; *hl = e - p;
    if (*hl && (*h)[*hl - 1] == '\r') (*hl)--;
    p = e + 1;
    e = p; while (e < f->size && f->data[e] != '\n') e++;
    *s = f->data + p; *sl = e - p;
    if (*sl && (*s)[*sl - 1] == '\r') (*sl)--;
    p = e + 1;
    if (*fasta) { *q = ""; *ql = 0; f->pos = p; return 1; }
    e = p; while (e < f->size && f->data[e] != '\n') e++;   /* '+' line */
    p = e + 1;
    e = p; while (e < f->size && f->data[e] != '\n') e++;
    *q = f->data + p; *ql = e - p;
    if (*ql && (*q)[*ql - 1] == '\r') (*ql)--;
    f->pos = e + 1;
    return 1;
}

co_reads* co_reads_from_files(const char* const* files, int nfiles, const co_opts* o) {
    infile in[2];
    memset(in, 0, sizeof(in));
    if (nfiles < 1 || nfiles > 2) return NULL;
    for (int i = 0; i < nfiles; i++)
        if (load_file(files[i], &in[i]) != 0) { fprintf(stderr, "care-oracle: cannot read %s\n", files[i]); return NULL; }

    sbuf text = {0};
    size_t cap = 1 << 16, n = 0;
    size_t* off = xmalloc(cap * sizeof(size_t));
    int32_t* lens = xmalloc(cap * sizeof(int32_t));
    int fasta = 0;
    /* two PE files are interleaved mate by mate (readlibraryio.hpp:130-170);
     * SE files are concatenated */
    int cur = 0;
    for (;;) {
        const char *h, *s, *q; size_t hl, sl, ql; int fa;
        int got = next_record(&in[cur], &h, &hl, &s, &sl, &q, &ql, &fa);
        if (!got) {
            if (nfiles == 2 && !o->paired_end && cur == 0) { cur = 1; continue; }
            break;
        }
        fasta |= fa;
        if (n == cap) {
            cap *= 2;
            off = realloc(off, cap * sizeof(size_t));
            lens = realloc(lens, cap * sizeof(int32_t));
        }
        off[n] = text.len;
        lens[n] = (int32_t)sl;
        sb_put(&text, h, hl); sb_put(&text, "", 1);
        sb_put(&text, s, sl); sb_put(&text, "", 1);
        sb_put(&text, q, ql); sb_put(&text, "", 1);
        n++;
        if (nfiles == 2 && o->paired_end) cur ^= 1;
    }
    for (int i = 0; i < nfiles; i++) free(in[i].data);

    co_reads* r = xcalloc(1, sizeof(co_reads));
    r->n = (uint32_t)n;
    r->text = text.buf;
    r->rec_off = off;
    r->len = lens;
    r->fasta = fasta;
    r->quality_bits = o->quality_bits;
    /* main_correct_cpu.cpp:103-117: no quality scores in input -> disabled */
    r->has_quality = o->use_quality && !fasta;
    int mn = 1 << 30, mx = 0;
    for (size_t i = 0; i < n; i++) { if (lens[i] < mn) mn = lens[i]; if (lens[i] > mx) mx = lens[i]; }
    if (n == 0) mn = 0;
    r->min_len = mn; r->max_len = mx;
    r->seq_pitch = ints2bit(mx);
    r->qual_pitch = qual_ints(mx, o->quality_bits);
    r->seq = xcalloc(n * (size_t)r->seq_pitch, 4);
    r->qual = r->has_quality ? xcalloc(n * (size_t)r->qual_pitch, 4) : NULL;
    r->ambig = xcalloc(n, 1);

    /* preprocessSequence (chunkedreadstorageconstruction.hpp:67-92): lower case
     * is upper-cased, any other character is replaced by A,C,G,T in rotation.
     * The rotation counter starts at 0 for every parser batch of 65536 reads
     * (:106, :259), and batches restart at each input file for SE input
     * (:371-386). */
    char* tmp = xmalloc((size_t)mx + 1);
    size_t fileStart = 0;
    int Ncount = 0;
    size_t secondFileFirst = (size_t)-1;
    if (nfiles == 2 && !o->paired_end) {
        /* find the first read of the second file: re-count records of file 0 */
        infile f0; load_file(files[0], &f0);
        size_t c0 = 0; const char *h, *s, *q; size_t hl, sl, ql; int fa;
        while (next_record(&f0, &h, &hl, &s, &sl, &q, &ql, &fa)) c0++;
        free(f0.data);
        secondFileFirst = c0;
    }
    for (size_t i = 0; i < n; i++) {
        if (i == secondFileFirst) fileStart = i;
        if ((i - fileStart) % 65536 == 0) Ncount = 0;
        const char* s = r->text + off[i];
        const size_t hl = strlen(s);
        s += hl + 1;
        const int L = lens[i];
        int und = 0;
        for (int p = 0; p < L; p++) {
            char c = s[p];
            if (c == 'a') c = 'A'; else if (c == 'c') c = 'C'; else if (c == 'g') c = 'G'; else if (c == 't') c = 'T';
            else if (c != 'A' && c != 'C' && c != 'G' && c != 'T') {
                und = 1;
                c = "ACGT"[Ncount];
                Ncount = (Ncount + 1) % 4;
            }
            tmp[p] = c;
        }
        r->ambig[i] = (uint8_t)und;
        co_encode_2bit(tmp, L, r->seq + i * (size_t)r->seq_pitch);
        if (r->has_quality) {
            const char* q = s + L + 1;
            co_encode_quality(q, L, o->quality_bits, r->qual + i * (size_t)r->qual_pitch);
        }
    }
    free(tmp);
    return r;
}

void co_reads_free(co_reads* r) {
    if (!r) return;
    free(r->seq); free(r->qual); free(r->len); free(r->ambig); free(r->text); free(r->rec_off);
    free(r);
}

/* ------------------------------------------------------------------ */
/* Hash tables: ordinaryminhasher.hpp:376-426 (insert),                 */
/* groupbykey.hpp:99-249 (group, sort values, clear buckets),           */
/* cpuhashtable.hpp:499-597 (lookup)                                    */
/* ------------------------------------------------------------------ */

typedef struct { uint64_t key; uint32_t id; } kv;
static int kv_cmp(const void* a, const void* b) {
    const kv* x = a; const kv* y = b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

typedef struct { const co_reads* r; const co_opts* o; co_tables* t; int h0, h1; uint64_t* sig; } build_job;

static void* build_tables_range(void* arg) {
    build_job* j = arg;
    const uint32_t n = j->r->n;
    kv* pairs = xmalloc((size_t)n * sizeof(kv));
    for (int h = j->h0; h < j->h1; h++) {
        for (uint32_t i = 0; i < n; i++) { pairs[i].key = j->sig[(size_t)i * j->t->num_maps + h]; pairs[i].id = i; }
        /* stable_sort_by_key over iota values == sort by (key, id) */
        qsort(pairs, n, sizeof(kv), kv_cmp);
        co_table* T = &j->t->t[h];
        size_t nk = 0, nv = 0;
        for (uint32_t i = 0; i < n;) {
            uint32_t e = i; while (e < n && pairs[e].key == pairs[i].key) e++;
            const uint32_t c = e - i;
            if (c >= 2 && (int)c <= j->t->threshold) { nk++; nv += c; }   /* :181-209 */
            i = e;
        }
        T->keys = xmalloc(nk * 8); T->offsets = xmalloc((nk + 1) * 4); T->values = xmalloc(nv * 4);
        T->nkeys = nk;
        size_t kk = 0, vv = 0;
        T->offsets[0] = 0;
        for (uint32_t i = 0; i < n;) {
            uint32_t e = i; while (e < n && pairs[e].key == pairs[i].key) e++;
            const uint32_t c = e - i;
            if (c >= 2 && (int)c <= j->t->threshold) {
                T->keys[kk] = pairs[i].key;
                for (uint32_t x = i; x < e; x++) T->values[vv++] = pairs[x].id;
                T->offsets[++kk] = (uint32_t)vv;
            }
            i = e;
        }
    }
    free(pairs);
    return NULL;
}

co_tables* co_build_tables(const co_reads* r, const co_opts* o) {
    co_tables* t = xcalloc(1, sizeof(co_tables));
    t->num_maps = o->num_maps;
    t->k = o->kmerlength;
    t->threshold = co_threshold(o->estimated_coverage);
    t->t = xcalloc((size_t)o->num_maps, sizeof(co_table));
    uint64_t* sig = xmalloc((size_t)r->n * o->num_maps * 8);
    /* every read is inserted, short ones too (their key is the all-ones mask) */
    for (uint32_t i = 0; i < r->n; i++)
        co_signature(r->seq + (size_t)i * r->seq_pitch, r->len[i], o->kmerlength, o->num_maps,
                     sig + (size_t)i * o->num_maps);
    int nt = o->threads > 0 ? o->threads : 1;
    if (nt > o->num_maps) nt = o->num_maps;
    pthread_t th[64];
    build_job jobs[64];
    if (nt > 64) nt = 64;
    for (int i = 0; i < nt; i++) {
        jobs[i] = (build_job){r, o, t, o->num_maps * i / nt, o->num_maps * (i + 1) / nt, sig};
        pthread_create(&th[i], NULL, build_tables_range, &jobs[i]);
    }
    for (int i = 0; i < nt; i++) pthread_join(th[i], NULL);
    free(sig);
    return t;
}

void co_tables_free(co_tables* t) {
    if (!t) return;
    for (int h = 0; h < t->num_maps; h++) { free(t->t[h].keys); free(t->t[h].offsets); free(t->t[h].values); }
    free(t->t); free(t);
}

/* CpuReadOnlyMultiValueHashTable::query (cpuhashtable.hpp:576-597) +
 * OrdinaryCpuMinhasher::queryMap (ordinaryminhasher.hpp:437-449) */
static const uint32_t* table_query(const co_table* T, uint64_t key, int threshold, int* cnt) {
    size_t lo = 0, hi = T->nkeys;
    while (lo < hi) { size_t m = (lo + hi) / 2; if (T->keys[m] < key) lo = m + 1; else hi = m; }
    if (lo < T->nkeys && T->keys[lo] == key) {
        const int c = (int)(T->offsets[lo + 1] - T->offsets[lo]);
        if (c > threshold) { *cnt = 0; return NULL; }
        *cnt = c;
        return T->values + T->offsets[lo];
    }
    *cnt = 0;
    return NULL;
}

/* ------------------------------------------------------------------ */
/* Shifted Hamming distance: src/cpu_alignment.cpp:32-323,              */
/* include/cpu_alignment.hpp:411-464                                    */
/* ------------------------------------------------------------------ */

static int popc(uint32_t x) { return __builtin_popcount(x); }

/* hammingDistanceWithShiftNum, cpu_alignment.cpp:48-117 */
static int ham_shift(int shift_len, int ov, int max_errors,
                     const uint32_t* lhi, const uint32_t* llo,
                     const uint32_t* rhi, const uint32_t* rlo) {
    if (shift_len < 0) shift_len = -shift_len;
    if (ov == 0) return max_errors + 1;
    const int parts = (ov + 31) >> 5;
    const int rem = (parts << 5) - ov;
    const int ps = shift_len >> 5, bs = shift_len & 31;
    int result = 0;
    for (int i = 0; i < parts - 1 && result < max_errors; i++) {
        uint32_t A1 = lhi[i + ps] << bs, A2 = llo[i + ps] << bs;
        uint32_t B1 = bs ? lhi[i + ps + 1] >> (32 - bs) : 0;
        uint32_t B2 = bs ? llo[i + ps + 1] >> (32 - bs) : 0;
        result += popc(((A1 | B1) ^ rhi[i]) | ((A2 | B2) ^ rlo[i]));
    }
    if (result >= max_errors) return result;
    const uint32_t mask = rem == 0 ? 0xFFFFFFFFu : 0xFFFFFFFFu << rem;
    const int i = parts - 1;
    uint32_t A1 = lhi[i + ps] << bs, A2 = llo[i + ps] << bs;
    uint32_t B1 = bs ? lhi[i + ps + 1] >> (32 - bs) : 0;
    uint32_t B2 = bs ? llo[i + ps + 1] >> (32 - bs) : 0;
    result += popc((((A1 | B1) ^ rhi[i]) | ((A2 | B2) ^ rlo[i])) & mask);
    return result;
}

/* cpuShiftedHammingDistancePopcount2BitHiLo, cpu_alignment.cpp:32-323 */
static void shd_hilo(const uint32_t* aHL, int la, const uint32_t* cHL, int lc,
                     int min_overlap, float maxErrorRate, float min_overlap_ratio, co_align* out) {
    const int aInts = ints2bithilo(la), cInts = ints2bithilo(lc);
    const int maxInts = (aInts + cInts) * 2;
    uint32_t buf[2 * 64 + 8];
    uint32_t* sbuf_ = maxInts <= (int)(sizeof(buf) / 4) ? buf : xmalloc((size_t)maxInts * 4);
    const uint32_t* aHi = aHL; const uint32_t* aLo = aHL + aInts / 2;
    const uint32_t* cHi = cHL; const uint32_t* cLo = cHL + cInts / 2;
    const int total = la + lc;
    const int minov = min_overlap > (int)((float)la * min_overlap_ratio) ? min_overlap : (int)((float)la * min_overlap_ratio);
    int bestScore = total, bestShift = -lc;

    /* handle_shift, :247-276 */
#define HANDLE(SHIFT, OV, LHI, LLO, RHI, RLO, BROKE) do { \
        int mex = (int)((float)(OV) * maxErrorRate); \
        const int lim2 = bestScore - total + 2 * (OV); \
        if (lim2 < mex) mex = lim2; \
        if (mex > 0) { \
            const int mm = ham_shift((SHIFT), (OV), mex, LHI, LLO, RHI, RLO); \
            const int sc = mm < mex ? mm + total - 2 * (OV) : 0x7fffffff; \
            if (sc < bestScore) { bestScore = sc; bestShift = (SHIFT); } \
        } else { BROKE = 1; } \
    } while (0)

    for (int i = 0; i < maxInts; i++) sbuf_[i] = 0;
    memcpy(sbuf_, aHi, (size_t)(aInts / 2) * 4);
    memcpy(sbuf_ + maxInts / 2, aLo, (size_t)(aInts / 2) * 4);
    for (int s = 0; s < la - minov + 1; ++s) {
        const int ov = (la - s) < lc ? (la - s) : lc;
        int broke = 0;
        HANDLE(s, ov, sbuf_, sbuf_ + maxInts / 2, cHi, cLo, broke);
        if (broke) break;
    }
    for (int i = 0; i < maxInts; i++) sbuf_[i] = 0;
    memcpy(sbuf_, cHi, (size_t)(cInts / 2) * 4);
    memcpy(sbuf_ + maxInts / 2, cLo, (size_t)(cInts / 2) * 4);
    for (int s = -1; s >= -lc + minov; --s) {
        const int ov = la < (lc + s) ? la : (lc + s);
        int broke = 0;
        HANDLE(s, ov, sbuf_, sbuf_ + maxInts / 2, aHi, aLo, broke);
        if (broke) break;
    }
#undef HANDLE
    if (sbuf_ != buf) free(sbuf_);
    out->valid = bestShift != -lc;
    const int cb = -bestShift > 0 ? -bestShift : 0;
    const int ce = lc < la - bestShift ? lc : la - bestShift;
    const int ovs = ce - cb;
    out->score = bestScore;
    out->overlap = ovs;
    out->shift = bestShift;
    out->nops = bestScore - total + 2 * ovs;
}

void co_shd(const uint32_t* anchor2bit, int la, const uint32_t* cand2bit, int lc,
            int min_overlap, float max_error_rate, float min_overlap_ratio, co_align* out) {
    uint32_t ah[64], ch[64];
    co_to_hilo(anchor2bit, la, ah);
    co_to_hilo(cand2bit, lc, ch);
    shd_hilo(ah, la, ch, lc, min_overlap, max_error_rate, min_overlap_ratio, out);
}

/* chooseBestAlignmentOrientation, alignmentorientation.hpp:12-92.
 * Returns 1 = Forward, 2 = ReverseComplement, 3 = None. */
int co_orientation(const co_align* f, const co_align* r, int la, int lc,
                   float min_overlap_ratio, int min_overlap, float estimated_errorrate) {
    const float maxErrorRate = estimated_errorrate * 4.0f;
    int ret = 3;
    const int mo = (int)(la * min_overlap_ratio) > min_overlap ? (int)(la * min_overlap_ratio) : min_overlap;
    if (f->valid && f->overlap >= mo) {
        if (r->valid && r->overlap >= mo) {
            const float ratio = (float)f->nops / f->overlap;
            const float rratio = (float)r->nops / r->overlap;
            if (ratio < rratio) { if (ratio < maxErrorRate) ret = 1; }
            else if (rratio < ratio) { if (rratio < maxErrorRate) ret = 2; }
            else if (ratio < maxErrorRate) ret = f->overlap > r->overlap ? 1 : 2;
        } else if ((float)f->nops / f->overlap < maxErrorRate) ret = 1;
    } else if (r->valid && r->overlap >= mo) {
        if ((float)r->nops / r->overlap < maxErrorRate) ret = 2;
    }
    (void)lc;
    return ret;
}

/* findPositionsOfPairedReadIds -> flagPairedCandidates, util.hpp:1016-1197.
 * Both lists sorted ascending; reads x,y are mates iff x/2 == y/2. */
void co_pair_flags(const uint32_t* l1, int n1, const uint32_t* l2, int n2, uint8_t* f1, uint8_t* f2) {
    memset(f1, 0, (size_t)n1); memset(f2, 0, (size_t)n2);
    int a = 0, b = 0;
    while (a < n1 && b < n2) {
        const int e1 = (a + 1 < n1 && l1[a] / 2 == l1[a + 1] / 2) ? 2 : 1;
        const int e2 = (b + 1 < n2 && l2[b] / 2 == l2[b + 1] / 2) ? 2 : 1;
        const int same = l1[a] / 2 == l2[b] / 2;
        if (e1 == 1 && e2 == 1) {
            if (same) {
                if (l1[a] != l2[b]) { f1[a] = 1; f2[b] = 1; }
                a++; b++;
            } else if (l1[a] < l2[b]) a++; else b++;
        } else if (e1 == 2 && e2 == 2) {
            if (same) { f1[a] = f1[a + 1] = 1; f2[b] = f2[b + 1] = 1; a += 2; b += 2; }
            else if (l1[a] < l2[b]) a += 2; else b += 2;
        } else if (e1 == 2 && e2 == 1) {
            if (same) {
                if (l1[a] == l2[b]) { f1[a + 1] = 1; f2[b] = 1; }
                else { f1[a] = 1; f2[b] = 1; }
                a += 2; b += 1;
            } else if (l1[a] < l2[b]) a += 2; else b += 1;
        } else {
            if (same) {
                if (l1[a] == l2[b]) { f1[a] = 1; f2[b + 1] = 1; }
                else { f1[a] = 1; f2[b] = 1; }
                a += 1; b += 2;
            } else if (l1[a] < l2[b]) a += 1; else b += 2;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Float compares, include/hostdevicefunctions.cuh:9-29                 */
/* ------------------------------------------------------------------ */
static int feq(float l, float r) { const float d = l - r < 0 ? -(l - r) : l - r; return d < 1e-5f; }
static int fleq(float l, float r) { return (l < r) || feq(l, r); }
static int fgeq(float l, float r) { return (l > r) || feq(l, r); }

/* calculateOverlapWeight, hostdevicefunctions.cuh:93-97 */
static float overlap_weight(int nops, int overlap, float maxMismatchRatio) {
    return 1.0f - sqrtf(nops / (overlap * maxMismatchRatio));
}

/* ------------------------------------------------------------------ */
/* Per-anchor task state (include/cpucorrectortask.hpp:28-56)           */
/* ------------------------------------------------------------------ */

typedef struct {
    int cap, cols_cap;
    /* candidates */
    int n;
    uint32_t* ids;
    uint32_t* seq;      /* oriented 2-bit, pitch */
    uint32_t* rcseq;
    int* len;
    co_align* al;
    co_align* ral;
    int* flag;
    uint8_t* paired;
    char* quals;        /* qpitch chars per candidate (oriented) */
    char* dec;          /* decoded oriented candidate, dpitch */
    int* shifts; int* ops; int* ovs; float* w;
    uint8_t* remove;
    /* msa */
    int ncols, abegin, aend;
    int *cA, *cC, *cG, *cT, *cov, *origCov;
    float *wA, *wC, *wG, *wT, *support, *origW;
    char* cons;
    /* anchor */
    char* anchor_dec;
    char* anchor_q;
    char* fwdunc;
    uint32_t hiloA[64];
    uint32_t hiloC[64];
    float qw[256];
} task_t;

static void task_init(task_t* t, int cap, int maxlen, int seq_pitch) {
    memset(t, 0, sizeof(*t));
    t->cap = cap;
    t->ids = xmalloc((size_t)cap * 4);
    t->seq = xmalloc((size_t)cap * seq_pitch * 4);
    t->rcseq = xmalloc((size_t)cap * seq_pitch * 4);
    t->len = xmalloc((size_t)cap * 4);
    t->al = xmalloc((size_t)cap * sizeof(co_align));
    t->ral = xmalloc((size_t)cap * sizeof(co_align));
    t->flag = xmalloc((size_t)cap * 4);
    t->paired = xmalloc((size_t)cap);
    t->quals = xmalloc((size_t)cap * maxlen);
    t->dec = xmalloc((size_t)cap * maxlen);
    t->shifts = xmalloc((size_t)cap * 4);
    t->ops = xmalloc((size_t)cap * 4);
    t->ovs = xmalloc((size_t)cap * 4);
    t->w = xmalloc((size_t)cap * 4);
    t->remove = xmalloc((size_t)cap);
    const int cc = 3 * maxlen + 8;
    t->cols_cap = cc;
    t->cA = xmalloc(cc * 4); t->cC = xmalloc(cc * 4); t->cG = xmalloc(cc * 4); t->cT = xmalloc(cc * 4);
    t->cov = xmalloc(cc * 4); t->origCov = xmalloc(cc * 4);
    t->wA = xmalloc(cc * 4); t->wC = xmalloc(cc * 4); t->wG = xmalloc(cc * 4); t->wT = xmalloc(cc * 4);
    t->support = xmalloc(cc * 4); t->origW = xmalloc(cc * 4);
    t->cons = xmalloc(cc);
    t->anchor_dec = xmalloc((size_t)maxlen + 1);
    t->anchor_q = xmalloc((size_t)maxlen + 1);
    t->fwdunc = xmalloc((size_t)maxlen + 1);
    co_quality_weights(t->qw);
}

static void task_free(task_t* t) {
    free(t->ids); free(t->seq); free(t->rcseq); free(t->len); free(t->al); free(t->ral); free(t->flag);
    free(t->paired); free(t->quals); free(t->dec); free(t->shifts); free(t->ops); free(t->ovs); free(t->w);
    free(t->remove); free(t->cA); free(t->cC); free(t->cG); free(t->cT); free(t->cov); free(t->origCov);
    free(t->wA); free(t->wC); free(t->wG); free(t->wT); free(t->support); free(t->origW); free(t->cons);
    free(t->anchor_dec); free(t->anchor_q); free(t->fwdunc);
}

typedef struct { const co_reads* r; const co_tables* tb; const co_opts* o; } ctx_t;

static int u32cmp(const void* a, const void* b) {
    const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : (x > y);
}

/* determineCandidateReadIds, corrector.hpp:571-650: query all maps, concat,
 * sort, unique, remove self, remove ambiguous. Returns the count. */
static int candidate_ids(const ctx_t* c, uint32_t anchor, uint32_t* out, int cap) {
    const co_reads* r = c->r;
    if (c->o->exclude_ambiguous && r->ambig[anchor]) return 0;
    const int L = r->len[anchor];
    int n = 0;
    if (L >= c->tb->k) {
        uint64_t sig[64];
        co_signature(r->seq + (size_t)anchor * r->seq_pitch, L, c->tb->k, c->tb->num_maps, sig);
        for (int h = 0; h < c->tb->num_maps; h++) {
            int cnt;
            const uint32_t* v = table_query(&c->tb->t[h], sig[h], c->tb->threshold, &cnt);
            for (int i = 0; i < cnt && n < cap; i++) out[n++] = v[i];
        }
    }
    qsort(out, (size_t)n, 4, u32cmp);
    int u = 0;
    for (int i = 0; i < n; i++) if (u == 0 || out[u - 1] != out[i]) out[u++] = out[i];
    int m = 0;
    for (int i = 0; i < u; i++) {
        if (out[i] == anchor) continue;
        if (c->o->exclude_ambiguous && r->ambig[out[i]]) continue;
        out[m++] = out[i];
    }
    return m;
}

/* ---- MSA: src/msa.cpp ---- */

/* MultipleSequenceAlignment::build / addSequence / findConsensus /
 * findOrigWeightAndCoverage, msa.cpp:9-173 */
static void msa_build(task_t* t, const ctx_t* c, int la) {
    const int dp = c->r->max_len;
    int start = 0, end = la;
    for (int i = 0; i < t->n; i++) {
        const int e = t->len[i] + t->shifts[i];
        if (t->shifts[i] < start) start = t->shifts[i];
        if (e > end) end = e;
    }
    t->ncols = end - start;
    t->abegin = -start > 0 ? -start : 0;
    t->aend = t->abegin + la;
    const int nc = t->ncols;
    memset(t->cA, 0, nc * 4); memset(t->cC, 0, nc * 4); memset(t->cG, 0, nc * 4); memset(t->cT, 0, nc * 4);
    memset(t->cov, 0, nc * 4); memset(t->origCov, 0, nc * 4);
    for (int i = 0; i < nc; i++) { t->wA[i] = t->wC[i] = t->wG[i] = t->wT[i] = 0.0f; t->support[i] = 0.0f; t->origW[i] = 0.0f; }
    const int useQ = c->o->use_quality && c->r->has_quality;
    for (int s = -1; s < t->n; s++) {
        const char* seq = s < 0 ? t->anchor_dec : t->dec + (size_t)s * dp;
        const char* q = s < 0 ? t->anchor_q : t->quals + (size_t)s * dp;
        const int L = s < 0 ? la : t->len[s];
        const int sh = s < 0 ? 0 : t->shifts[s];
        const float f = s < 0 ? 1.0f : t->w[s];
        for (int i = 0; i < L; i++) {                          /* addSequence :93-112 */
            const int g = t->abegin + sh + i;
            const float wgt = f * (useQ ? t->qw[(unsigned char)q[i]] : 1.0f);
            switch (seq[i]) {
                case 'A': t->cA[g]++; t->wA[g] += wgt; break;
                case 'C': t->cC[g]++; t->wC[g] += wgt; break;
                case 'G': t->cG[g]++; t->wG[g] += wgt; break;
                case 'T': t->cT[g]++; t->wT[g] += wgt; break;
            }
            t->cov[g]++;
        }
    }
    for (int col = 0; col < nc; col++) {                       /* findConsensus :135-157 */
        char cs = 'A'; float cw = t->wA[col];
        if (t->wC[col] > cw) { cs = 'C'; cw = t->wC[col]; }
        if (t->wG[col] > cw) { cs = 'G'; cw = t->wG[col]; }
        if (t->wT[col] > cw) { cs = 'T'; cw = t->wT[col]; }
        t->cons[col] = cs;
        const float colw = t->wA[col] + t->wC[col] + t->wG[col] + t->wT[col];
        t->support[col] = cw / colw;
    }
    for (int col = t->abegin; col < t->aend; col++) {          /* :159-173 */
        switch (t->anchor_dec[col - t->abegin]) {
            case 'A': t->origW[col] = t->wA[col]; t->origCov[col] = t->cA[col]; break;
            case 'C': t->origW[col] = t->wC[col]; t->origCov[col] = t->cC[col]; break;
            case 'G': t->origW[col] = t->wG[col]; t->origCov[col] = t->cG[col]; break;
            case 'T': t->origW[col] = t->wT[col]; t->origCov[col] = t->cT[col]; break;
        }
    }
}

/* findCandidatesOfDifferentRegion, msa.cpp:532-734. Returns 1 if a column
 * was found (performedMinimization); t->remove holds the verdicts. */
static int msa_different_region(task_t* t, int la, int dataset_coverage, int dp) {
    int mism = 0;
    for (int i = 0; i < la; i++) if (t->anchor_dec[i] != t->cons[t->abegin + i]) { mism = 1; break; }
    if (!mism) return 0;
    int found = 0, col = 0, foundIdx = 0;
    char foundBase = 'F';
    for (int ci = t->abegin; ci < t->aend && !found; ci++) {
        const int counts[4] = {t->cA[ci], t->cC[ci], t->cG[ci], t->cT[ci]};
        int consIdx = -1;
        switch (t->cons[ci]) { case 'A': consIdx = 0; break; case 'C': consIdx = 1; break; case 'G': consIdx = 2; break; case 'T': consIdx = 3; break; }
        int sig = -1;
        for (int b = 0; b < 4; b++)
            if (b != consIdx && (int)(dataset_coverage * 0.3f) <= counts[b]) sig = b;
        if (sig != -1) { found = 1; col = ci; foundBase = "ACGT"[sig]; foundIdx = sig; }
    }
    (void)foundIdx;
    if (!found) return 0;
    const char orig = t->anchor_dec[col - t->abegin];
    const int keepMatching = orig == foundBase;
    for (int i = 0; i < t->n; i++) {
        const int rb = t->abegin + t->shifts[i];
        const int re = rb + t->len[i];
        const int notAff = col < rb || re <= col;
        const char base = notAff ? 'F' : t->dec[(size_t)i * dp + (col - rb)];
        if (notAff) t->remove[i] = 0;
        else if (keepMatching && base == foundBase) t->remove[i] = 0;
        else if (!keepMatching && base != foundBase) t->remove[i] = 0;
        else t->remove[i] = 1;
    }
    int veryGood = 0;
    for (int i = 0; i < t->n; i++) if (t->remove[i] && t->w[i] >= 0.90f) veryGood = 1;
    if (veryGood) memset(t->remove, 0, (size_t)t->n);
    return 1;
}

/* compaction of all per-candidate arrays by a keep predicate (the
 * erase/copy_n blocks of corrector.hpp:982-1421) */
static void compact(task_t* t, const uint8_t* keep, int sp, int dp, int with_msa_arrays) {
    int w = 0;
    for (int i = 0; i < t->n; i++) {
        if (!keep[i]) continue;
        if (w != i) {
            t->ids[w] = t->ids[i];
            memcpy(t->seq + (size_t)w * sp, t->seq + (size_t)i * sp, (size_t)sp * 4);
            memcpy(t->rcseq + (size_t)w * sp, t->rcseq + (size_t)i * sp, (size_t)sp * 4);
            t->len[w] = t->len[i]; t->al[w] = t->al[i]; t->ral[w] = t->ral[i];
            t->flag[w] = t->flag[i]; t->paired[w] = t->paired[i];
            if (with_msa_arrays) {
                memcpy(t->quals + (size_t)w * dp, t->quals + (size_t)i * dp, (size_t)dp);
                memcpy(t->dec + (size_t)w * dp, t->dec + (size_t)i * dp, (size_t)dp);
                t->shifts[w] = t->shifts[i]; t->ops[w] = t->ops[i]; t->ovs[w] = t->ovs[i]; t->w[w] = t->w[i];
            }
        }
        w++;
    }
    t->n = w;
}

/* ------------------------------------------------------------------ */
/* Learned decision columns. The reference's classifier hook asks, for  */
/* every anchor column of a non-HQ MSA whose original base differs from  */
/* the consensus, whether the consensus base should be written          */
/* (correctAnchorClf, corrector.hpp:1448-1472; features in the spirit   */
/* of extract_anchor_v3, classification.hpp:748-797, widened to 24).    */
/* ------------------------------------------------------------------ */

/* float -> bfloat16 -> float, round to nearest even */
float co_bf16_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return x;          /* NaN */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

static float gelu_f(float x) { return (0.5f * x) * (1.0f + erff(x * 0.70710678118654752f)); }

/* Forward pass with the device path's roundings: normalised inputs,
 * weights and hidden activations are bfloat16 values; products and sums
 * are FP32 (sums here run in index order). */
float co_mlp_logit(const float* P, const float* x) {
    float xn[CO_NFEAT], h1[CO_HIDDEN];
    for (int k = 0; k < CO_NFEAT; k++) xn[k] = co_bf16_round((x[k] - P[CO_MLP_MEAN + k]) * P[CO_MLP_ISTD + k]);
    for (int n = 0; n < CO_HIDDEN; n++) {
        float z = 0.0f;
        for (int k = 0; k < CO_NFEAT; k++) z += xn[k] * co_bf16_round(P[CO_MLP_W1 + n * CO_NFEAT + k]);
        h1[n] = co_bf16_round(gelu_f(z + P[CO_MLP_B1 + n]));
    }
    float s = 0.0f;
    for (int n = 0; n < CO_HIDDEN; n++) {
        float z = 0.0f;
        for (int k = 0; k < CO_HIDDEN; k++) z += h1[k] * co_bf16_round(P[CO_MLP_W2 + n * CO_HIDDEN + k]);
        const float h2 = co_bf16_round(gelu_f(z + P[CO_MLP_B2 + n]));
        s += h2 * co_bf16_round(P[CO_MLP_W3 + n]);
    }
    return s + P[CO_MLP_B3];
}

typedef struct {
    int allGood, minCov, maxCov, nmis;
    float avgSup, minSup;
} clf_anchor;

static int code_of(char b) { return b == 'A' ? 0 : b == 'C' ? 1 : b == 'G' ? 2 : 3; }

/* the 24 features of anchor position p; every float operation in the
 * order the device code performs it */
static void clf_features(const task_t* t, const ctx_t* c, int la, int p, const clf_anchor* A, float* x) {
    const co_opts* o = c->o;
    const int useQ = o->use_quality && c->r->has_quality;
    const int col = t->abegin + p;
    const float E = o->estimated_coverage;
    const int cb = code_of(t->cons[col]);
    const int cnt[4] = {t->cA[col], t->cC[col], t->cG[col], t->cT[col]};
    const float w[4] = {t->wA[col], t->wC[col], t->wG[col], t->wT[col]};
    const float wsum = ((w[0] + w[1]) + w[2]) + w[3];
    const float wc = w[cb];
    const float wo = t->origW[col];
    const int oc = t->origCov[col];
    const int cc = cnt[cb];
    const float cov = (float)t->cov[col];
    x[0] = (float)oc / cov;
    x[1] = wo / wsum;
    x[2] = wo / (float)oc;
    x[3] = (float)cc / cov;
    x[4] = t->support[col];
    x[5] = wc / (float)cc;
    x[6] = wsum / cov;
    x[7] = cov / E;
    x[8] = wsum / E;
    x[9] = A->avgSup;
    x[10] = A->minSup;
    x[11] = (float)A->maxCov / E;
    x[12] = (float)A->minCov / E;
    x[13] = useQ ? t->qw[(unsigned char)t->anchor_q[p]] : 1.0f;
    x[14] = (float)(p < la - 1 - p ? p : la - 1 - p) / (float)la;
    x[15] = ((wsum - wc) - wo) / wsum;
    const int lo = p - 3 > 0 ? p - 3 : 0, hi = p + 3 < la - 1 ? p + 3 : la - 1;
    float ssum = 0.0f, smin = t->support[t->abegin + lo], qsum = 0.0f;
    for (int q = lo; q <= hi; q++) {
        const float sv = t->support[t->abegin + q];
        ssum += sv;
        if (sv < smin) smin = sv;
        qsum += useQ ? t->qw[(unsigned char)t->anchor_q[q]] : 1.0f;
    }
    const float nwin = (float)(hi - lo + 1);
    x[16] = ssum / nwin;
    x[17] = smin;
    x[18] = (float)A->nmis / (float)la;
    int nloc = 0;
    const int lo5 = p - 5 > 0 ? p - 5 : 0, hi5 = p + 5 < la - 1 ? p + 5 : la - 1;
    for (int q = lo5; q <= hi5; q++)
        if (q != p && t->anchor_dec[q] != t->cons[t->abegin + q]) nloc++;
    x[19] = (float)nloc / 10.0f;
    x[20] = (float)t->n / E;
    x[21] = A->allGood ? 1.0f : 0.0f;
    x[22] = (A->allGood || (t->support[col] > 0.90f && oc <= 2)) ? 1.0f : 0.0f;
    x[23] = qsum / nwin;
}

static void push_feature(co_results* res, const co_feature* f) {
    if (res->num_feats == res->cap_feats) {
        res->cap_feats = res->cap_feats ? res->cap_feats * 2 : 256;
        res->feats = realloc(res->feats, res->cap_feats * sizeof(co_feature));
    }
    res->feats[res->num_feats++] = *f;
}

/* decision columns of one corrected non-HQ anchor; in clf_mode 2 the
 * network's verdict replaces the plain rule's base in corr */
static void clf_columns(const ctx_t* c, const task_t* t, int la, uint32_t anchor, const clf_anchor* A,
                        char* corr, co_results* res) {
    const co_opts* o = c->o;
    for (int p = 0; p < la; p++) {
        const int col = t->abegin + p;
        const char ob = t->anchor_dec[p], cb = t->cons[col];
        if (ob == cb || t->cov[col] < o->clf_min_coverage) continue;
        co_feature f;
        memset(&f, 0, sizeof(f));
        f.read_id = anchor;
        f.pos = (int16_t)p;
        f.orig = (uint8_t)code_of(ob);
        f.cons = (uint8_t)code_of(cb);
        clf_features(t, c, la, p, A, f.x);
        if (o->clf_mode == 2) {
            f.logit = co_mlp_logit(o->mlp, f.x);
            corr[p] = f.logit > 0.0f ? cb : ob;
        }
        push_feature(res, &f);
    }
}

typedef struct {
    int corrected, hq;
    /* candidate corrections, indices into the final candidate list */
    int ncorr;
} anchor_out;

/* correction of one anchor whose candidate ids (and pair flags) are known:
 * the per-anchor body of CpuErrorCorrector::process / processMulti,
 * corrector.hpp:145-312 and :367-505. Writes into res. Also fills tr. */
static void correct_one(const ctx_t* c, task_t* t, uint32_t anchor, co_results* res, co_trace* tr) {
    const co_reads* r = c->r;
    const co_opts* o = c->o;
    const int sp = r->seq_pitch, dp = r->max_len;
    const uint32_t* aseq = r->seq + (size_t)anchor * sp;
    const int la = r->len[anchor];
    const size_t ai = anchor - res->first;
    co_anchor_result* AR = &res->anchors[ai];
    memset(AR, 0, sizeof(*AR));
    if (tr) { memset(tr, 0, sizeof(*tr)); tr->n_initial = t->n; }
    if (t->n == 0) return;

    co_decode_2bit(aseq, la, t->anchor_dec);
    const int useQ = o->use_quality && r->has_quality;
    if (useQ) co_decode_quality(r->qual + (size_t)anchor * r->qual_pitch, dp, r->quality_bits, t->anchor_q);

    /* getCandidateSequenceData + computeReverseComplementCandidates :880-922 */
    for (int i = 0; i < t->n; i++) {
        const uint32_t id = t->ids[i];
        t->len[i] = r->len[id];
        memcpy(t->seq + (size_t)i * sp, r->seq + (size_t)id * sp, (size_t)sp * 4);
        co_revcomp_2bit(t->seq + (size_t)i * sp, t->len[i], t->rcseq + (size_t)i * sp);
    }
    /* getCandidateAlignments :925-979 */
    co_to_hilo(aseq, la, t->hiloA);
    for (int i = 0; i < t->n; i++) {
        co_to_hilo(t->seq + (size_t)i * sp, t->len[i], t->hiloC);
        shd_hilo(t->hiloA, la, t->hiloC, t->len[i], o->min_overlap, o->max_error_rate, o->min_overlap_ratio, &t->al[i]);
    }
    for (int i = 0; i < t->n; i++) {
        co_to_hilo(t->rcseq + (size_t)i * sp, t->len[i], t->hiloC);
        shd_hilo(t->hiloA, la, t->hiloC, t->len[i], o->min_overlap, o->max_error_rate, o->min_overlap_ratio, &t->ral[i]);
    }
    for (int i = 0; i < t->n; i++)
        t->flag[i] = co_orientation(&t->al[i], &t->ral[i], la, t->len[i], o->min_overlap_ratio, o->min_overlap, o->estimated_errorrate);

    /* filterCandidatesByAlignmentFlag :982-1050: keep the chosen orientation */
    for (int i = 0; i < t->n; i++) {
        t->remove[i] = t->flag[i] != 3;
        if (t->flag[i] == 2) {
            memcpy(t->seq + (size_t)i * sp, t->rcseq + (size_t)i * sp, (size_t)sp * 4);
            t->al[i] = t->ral[i];
        }
    }
    compact(t, t->remove, sp, dp, 0);
    if (tr) tr->n_after_flag = t->n;
    if (t->n == 0) return;

    /* filterCandidatesByAlignmentMismatchRatio :1053-1211 */
    if (o->paired_end) {
        for (int i = 0; i < t->n; i++) {
            const float mr = (float)t->al[i].nops / (float)t->al[i].overlap;
            t->remove[i] = t->paired[i] || mr < o->paired_filter_threshold;
        }
    } else {
        const float base = o->estimated_errorrate * 1.0f;
        const float good = o->estimated_coverage * o->m_coverage;
        int cnt[3] = {0, 0, 0};
        for (int i = 0; i < t->n; i++) {
            const float mr = (float)t->al[i].nops / (float)t->al[i].overlap;
            if (mr < 2 * base) cnt[0]++;
            if (mr < 3 * base) cnt[1]++;
            if (mr < 4 * base) cnt[2]++;
        }
        float thr = -3.402823466e+38f;
        if (cnt[0] > 0 || cnt[1] > 0 || cnt[2] > 0) {
            if (cnt[0] >= good) thr = 2 * base;
            else if (cnt[1] >= good) thr = 3 * base;
            else if (cnt[2] >= good) thr = 4 * base;
        }
        for (int i = 0; i < t->n; i++) {
            const float mr = (float)t->al[i].nops / (float)t->al[i].overlap;
            t->remove[i] = mr < thr;
        }
    }
    compact(t, t->remove, sp, dp, 0);
    if (tr) tr->n_after_ratio = t->n;
    if (t->n == 0) return;

    /* qualities (:1214-1239): whole pitch decoded, reversed over the whole
     * pitch for reverse-complement alignments */
    for (int i = 0; i < t->n; i++) {
        char* q = t->quals + (size_t)i * dp;
        if (useQ) {
            co_decode_quality(r->qual + (size_t)t->ids[i] * r->qual_pitch, dp, r->quality_bits, q);
            if (t->flag[i] == 2)
                for (int a = 0, b = dp - 1; a < b; a++, b--) { char x = q[a]; q[a] = q[b]; q[b] = x; }
        }
        co_decode_2bit(t->seq + (size_t)i * sp, t->len[i], t->dec + (size_t)i * dp);   /* :1242-1258 */
        t->shifts[i] = t->al[i].shift;                                               /* :1260-1280 */
        t->ops[i] = t->al[i].nops;
        t->ovs[i] = t->al[i].overlap;
        t->w[i] = overlap_weight(t->al[i].nops, t->al[i].overlap, o->max_error_rate);
    }

    msa_build(t, c, la);
    /* refineMSA :1307-1421 */
    for (int it = 0; it < 5; it++) {
        if (!msa_different_region(t, la, (int)o->estimated_coverage, dp)) break;
        for (int i = 0; i < t->n; i++) t->remove[i] = !t->remove[i];
        compact(t, t->remove, sp, dp, 1);
        msa_build(t, c, la);
    }
    if (tr) { tr->n_final = t->n; tr->n_columns = t->ncols; tr->anchor_col_begin = t->abegin; }

    /* getMSAProperties, msa.cpp:304-376 */
    const float e = o->estimated_errorrate;
    const float avgThr = 1.0f - 1.0f * e, minThr = 1.0f - 3.0f * e;
    const float covThr = o->m_coverage / 6.0f * o->estimated_coverage;
    const int fc = t->abegin, lc = t->aend, dist = lc - fc;
    float minSup = t->support[fc];
    for (int i = fc + 1; i < lc; i++) if (t->support[i] < minSup) minSup = t->support[i];
    float sum = 0.0f;
    for (int i = fc; i < lc; i++) sum += t->support[i];
    const float avgSup = sum / dist;
    int minCov = t->cov[fc], maxCov = t->cov[fc];
    for (int i = fc + 1; i < lc; i++) if (t->cov[i] < minCov) minCov = t->cov[i];
    for (int i = fc + 1; i < lc; i++) if (t->cov[i] > maxCov) maxCov = t->cov[i];
    int hq = 0;
    const int allGood = fgeq(avgSup, avgThr) && fgeq(minSup, minThr) && fgeq((float)minCov, covThr);
    if (allGood) {
        int smallest = 100;
        const int pct = (int)ceilf(e * 100.0f);
        for (int p = pct; p >= 0; p--) {
            const float fac = p / 100.0f;
            const float at = 1.0f - 1.0f * fac, mt = 1.0f - 3.0f * fac;
            if (fgeq(avgSup, at) && fgeq(minSup, mt)) smallest = p;
        }
        hq = fgeq((float)minCov, covThr) && fleq((float)smallest, pct * 0.5f);
    }

    /* getCorrectedAnchor, msa.cpp:379-453 */
    char* corr = res->anchor_seq + ai * (size_t)dp;
    if (t->n == 0) {
        AR->status = 0;
    } else {
        AR->status = 1;
        if (allGood) memcpy(corr, t->cons + t->abegin, (size_t)la);
        else
            for (int i = 0; i < la; i++)
                corr[i] = (t->support[t->abegin + i] > 0.90f && t->origCov[t->abegin + i] <= 2) ? t->cons[t->abegin + i] : t->anchor_dec[i];
        if (o->clf_mode && !hq) {
            clf_anchor A;
            A.allGood = allGood; A.minCov = minCov; A.maxCov = maxCov;
            A.avgSup = avgSup; A.minSup = minSup;
            A.nmis = 0;
            for (int i = 0; i < la; i++) A.nmis += t->anchor_dec[i] != t->cons[t->abegin + i];
            clf_columns(c, t, la, anchor, &A, corr, res);
        }
    }
    AR->hq = (uint8_t)hq;
    if (AR->status) {
        /* makeOutputOfTask, corrector.hpp:1648-1675 */
        if (!r->ambig[anchor]) {
            const int maxE = la / 7;
            int ed = 0;
            for (int i = 0; i < la && ed <= maxE; i++) if (corr[i] != t->anchor_dec[i]) ed++;
            AR->use_edits = ed <= maxE;
            int full = 0;
            for (int i = 0; i < la; i++) if (corr[i] != t->anchor_dec[i]) full++;
            AR->num_edits = AR->use_edits ? full : 0;
        } else {
            AR->use_edits = 0;
        }
    }

    /* correctCandidatesClassic -> getCorrectedCandidates, msa.cpp:457-522;
     * output conversion corrector.hpp:1679-1757 */
    if (hq && o->correct_candidates) {
        const int ncc = o->new_columns_to_correct;
        for (int i = 0; i < t->n; i++) {
            const int qb = t->abegin + t->shifts[i];
            const int L = t->len[i];
            const int qe = qb + L;
            if (!(t->abegin - ncc <= qb && qb <= t->abegin + ncc && qe <= t->aend + ncc)) continue;
            if (res->num_cands == res->cap_cands) {
                res->cap_cands = res->cap_cands ? res->cap_cands * 2 : 1024;
                res->cands = realloc(res->cands, res->cap_cands * sizeof(co_cand_result));
                res->cand_seq = realloc(res->cand_seq, res->cap_cands * (size_t)dp);
            }
            co_cand_result* CR = &res->cands[res->num_cands];
            char* out = res->cand_seq + res->num_cands * (size_t)dp;
            res->num_cands++;
            CR->read_id = t->ids[i];
            CR->anchor_id = anchor;
            CR->shift = t->shifts[i];
            CR->length = L;
            const char* unc = t->dec + (size_t)i * dp;
            char* fwdunc = t->fwdunc;
            if (t->flag[i] == 1) {
                memcpy(out, t->cons + qb, (size_t)L);
                memcpy(fwdunc, unc, (size_t)L);
            } else {
                revcomp_decoded(t->cons + qb, L, out);
                revcomp_decoded(unc, L, fwdunc);
            }
            if (!r->ambig[t->ids[i]]) {
                const int maxE = L / 7;
                int ed = 0;
                for (int p = 0; p < L && ed <= maxE; p++) if (out[p] != fwdunc[p]) ed++;
                CR->use_edits = ed <= maxE;
            } else CR->use_edits = 0;
        }
    }
}

typedef struct {
    const ctx_t* c; co_results* res; uint32_t a0, a1; int maxcand;
} corr_job;

static void* correct_range(void* arg) {
    corr_job* j = arg;
    const ctx_t* c = j->c;
    const co_reads* r = c->r;
    task_t t;
    task_init(&t, j->maxcand, r->max_len, r->seq_pitch);
    uint32_t* l2 = xmalloc((size_t)j->maxcand * 4);
    uint8_t* f2 = xmalloc((size_t)j->maxcand);
    if (!c->o->paired_end) {
        for (uint32_t a = j->a0; a < j->a1; a++) {
            t.n = candidate_ids(c, a, t.ids, j->maxcand);
            memset(t.paired, 0, (size_t)t.n);
            correct_one(c, &t, a, j->res, NULL);
        }
    } else {
        /* processMulti, corrector.hpp:325-513: pair flags across mates */
        for (uint32_t a = j->a0; a + 1 < j->a1 + 1 && a < j->a1; a += 2) {
            int n1 = candidate_ids(c, a, t.ids, j->maxcand);
            int n2 = candidate_ids(c, a + 1, l2, j->maxcand);
            co_pair_flags(t.ids, n1, l2, n2, t.paired, f2);
            t.n = n1;
            correct_one(c, &t, a, j->res, NULL);
            memcpy(t.ids, l2, (size_t)n2 * 4);
            memcpy(t.paired, f2, (size_t)n2);
            t.n = n2;
            correct_one(c, &t, a + 1, j->res, NULL);
        }
    }
    free(l2); free(f2);
    task_free(&t);
    return NULL;
}

static int max_candidates(const co_tables* tb) { return tb->num_maps * tb->threshold + 1; }

co_results* co_correct(const co_reads* r, const co_tables* tb, const co_opts* o,
                       uint32_t first, uint32_t count, int threads) {
    ctx_t c = {r, tb, o};
    co_results* res = xcalloc(1, sizeof(co_results));
    res->first = first;
    res->count = count;
    res->max_len = r->max_len;
    res->anchors = xcalloc(count, sizeof(co_anchor_result));
    res->anchor_seq = xcalloc((size_t)count * (r->max_len ? r->max_len : 1), 1);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (o->paired_end && (first % 2 || count % 2)) { fprintf(stderr, "care-oracle: PE ranges must be pair aligned\n"); return res; }
    /* split into pair-aligned ranges; each thread collects its own candidate
     * corrections, merged in anchor order afterwards */
    co_results* part = xcalloc((size_t)threads, sizeof(co_results));
    pthread_t th[256];
    corr_job jobs[256];
    for (int i = 0; i < threads; i++) {
        uint64_t b = first + (uint64_t)count * i / threads, e = first + (uint64_t)count * (i + 1) / threads;
        if (o->paired_end) { b &= ~1ull; e &= ~1ull; if (i == threads - 1) e = first + count; }
        part[i] = *res;
        part[i].cands = NULL; part[i].cand_seq = NULL; part[i].num_cands = part[i].cap_cands = 0;
        part[i].feats = NULL; part[i].num_feats = part[i].cap_feats = 0;
        jobs[i] = (corr_job){&c, &part[i], (uint32_t)b, (uint32_t)e, max_candidates(tb)};
        pthread_create(&th[i], NULL, correct_range, &jobs[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
    size_t tot = 0;
    for (int i = 0; i < threads; i++) tot += part[i].num_cands;
    res->cap_cands = res->num_cands = tot;
    res->cands = xmalloc((tot ? tot : 1) * sizeof(co_cand_result));
    res->cand_seq = xmalloc((tot ? tot : 1) * (size_t)(r->max_len ? r->max_len : 1));
    size_t w = 0;
    for (int i = 0; i < threads; i++) {
        memcpy(res->cands + w, part[i].cands, part[i].num_cands * sizeof(co_cand_result));
        memcpy(res->cand_seq + w * r->max_len, part[i].cand_seq, part[i].num_cands * (size_t)r->max_len);
        w += part[i].num_cands;
        free(part[i].cands); free(part[i].cand_seq);
    }
    size_t nf = 0;
    for (int i = 0; i < threads; i++) nf += part[i].num_feats;
    res->num_feats = res->cap_feats = nf;
    res->feats = xmalloc((nf ? nf : 1) * sizeof(co_feature));
    w = 0;
    for (int i = 0; i < threads; i++) {
        if (part[i].num_feats) memcpy(res->feats + w, part[i].feats, part[i].num_feats * sizeof(co_feature));
        w += part[i].num_feats;
        free(part[i].feats);
    }
    free(part);
    return res;
}

void co_results_free(co_results* res) {
    if (!res) return;
    free(res->anchors); free(res->anchor_seq); free(res->cands); free(res->cand_seq); free(res->feats); free(res);
}

int co_trace_anchor(const co_reads* r, const co_tables* tb, const co_opts* o,
                    uint32_t anchor, co_trace* tr,
                    uint32_t* ids, int* shifts, int* orient, float* weights, int cap,
                    uint32_t* initial_ids, int initial_cap) {
    ctx_t c = {r, tb, o};
    const int mc = max_candidates(tb);
    task_t t;
    task_init(&t, mc, r->max_len, r->seq_pitch);
    co_results res;
    memset(&res, 0, sizeof(res));
    res.first = anchor; res.count = 1; res.max_len = r->max_len;
    co_anchor_result ar;
    res.anchors = &ar;
    res.anchor_seq = xmalloc((size_t)r->max_len + 1);
    t.n = candidate_ids(&c, anchor, t.ids, mc);
    memset(t.paired, 0, (size_t)mc);
    if (o->paired_end) {
        const uint32_t mate = anchor ^ 1u;
        uint32_t* l2 = xmalloc((size_t)mc * 4);
        uint8_t* f2 = xmalloc((size_t)mc);
        const int n2 = candidate_ids(&c, mate, l2, mc);
        if (anchor % 2 == 0) co_pair_flags(t.ids, t.n, l2, n2, t.paired, f2);
        else co_pair_flags(l2, n2, t.ids, t.n, f2, t.paired);
        free(l2); free(f2);
    }
    for (int i = 0; i < t.n && i < initial_cap; i++) initial_ids[i] = t.ids[i];
    correct_one(&c, &t, anchor, &res, tr);
    for (int i = 0; i < t.n && i < cap; i++) {
        ids[i] = t.ids[i]; shifts[i] = t.shifts[i]; orient[i] = t.flag[i]; weights[i] = t.w[i];
    }
    free(res.anchor_seq); free(res.cands); free(res.cand_seq); free(res.feats);
    task_free(&t);
    return tr->n_final;
}

/* ------------------------------------------------------------------ */
/* Output: correct_cpu.cpp:255-291 (save filter),                       */
/* correctionresultoutput.cpp:730-1020 (combiner), readlibraryio.cpp    */
/* ------------------------------------------------------------------ */

typedef struct { uint32_t read; uint32_t idx; } cref;
static int cref_cmp(const void* a, const void* b) {
    const cref* x = a; const cref* y = b;
    if (x->read != y->read) return x->read < y->read ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* "materialize" a result as the sequence the combiner would write: edits
 * applied to the original read, or the stored full sequence */
static void materialize(const char* orig, const char* seq, const char* base_dec, int L, int use_edits, char* out) {
    if (use_edits) {
        memcpy(out, orig, (size_t)L);
        for (int i = 0; i < L; i++) if (seq[i] != base_dec[i]) out[i] = seq[i];
    } else memcpy(out, seq, (size_t)L);
}

int co_write_output(const co_reads* r, const co_results* res, const co_opts* o, const char* outfile) {
    FILE* fp = fopen(outfile, "wb");
    if (!fp) return -1;
    const int dp = r->max_len;
    const size_t nc = res->num_cands;
    cref* cr = xmalloc((nc ? nc : 1) * sizeof(cref));
    for (size_t i = 0; i < nc; i++) { cr[i].read = res->cands[i].read_id; cr[i].idx = (uint32_t)i; }
    qsort(cr, nc, sizeof(cref), cref_cmp);
    char* dec = xmalloc((size_t)dp + 1);
    char* m0 = xmalloc((size_t)dp + 1);
    char* m1 = xmalloc((size_t)dp + 1);
    char* outseq = xmalloc((size_t)dp + 1);
    /* mergeSerializedResultsWithOriginalReads_multithreaded (:30-440) calls the
     * combiner -- and appends a quality label -- only for reads up to the last
     * read id that has a stored result; later reads are copied unchanged.
     * Stored: anchor results passing the save filter, and candidate results
     * for reads that are not HQ anchors (a candidate result for an HQ anchor is
     * dropped once that anchor's flag is set, corrector.hpp:1682-1684). */
    int64_t last = -1;
    for (uint32_t k = 0; k < res->count; k++) {
        const co_anchor_result* A = &res->anchors[k];
        if (A->status == 1 && !(A->hq && A->use_edits && A->num_edits == 0)) last = (int64_t)(res->first + k) > last ? (int64_t)(res->first + k) : last;
    }
    for (size_t k = 0; k < nc; k++) {
        const uint32_t id = res->cands[k].read_id;
        const int hqAnchor = id >= res->first && id < res->first + res->count &&
                             res->anchors[id - res->first].status == 1 && res->anchors[id - res->first].hq;
        if (!hqAnchor && (int64_t)id > last) last = id;
    }
    size_t ci = 0;
    for (uint32_t i = 0; i < r->n; i++) {
        const char* h = r->text + r->rec_off[i];
        const char* s = h + strlen(h) + 1;
        const char* q = s + strlen(s) + 1;
        const int L = r->len[i];
        memcpy(outseq, s, (size_t)L);
        int corrected = 0, label = 0;
        size_t cb = ci;
        while (ci < nc && cr[ci].read == i) ci++;
        const size_t ncand = ci - cb;
        int hasA = 0;
        const co_anchor_result* A = NULL;
        if (i >= res->first && i < res->first + res->count) {
            A = &res->anchors[i - res->first];
            /* saved iff corrected and not (hq && useEdits && 0 edits) */
            hasA = A->status == 1 && !(A->hq && A->use_edits && A->num_edits == 0);
        }
        if (hasA) {
            const char* aseq = res->anchor_seq + (size_t)(i - res->first) * dp;
            co_decode_2bit(r->seq + (size_t)i * r->seq_pitch, L, dec);
            if (A->hq) {
                materialize(s, aseq, dec, L, A->use_edits, outseq);
                corrected = 1; label = 3;
            } else if (1 + ncand >= 3) {
                materialize(s, aseq, dec, L, A->use_edits, m0);
                int same = 1;
                for (size_t k = cb; k < ci && same; k++) {
                    const co_cand_result* C = &res->cands[cr[k].idx];
                    const char* cs = res->cand_seq + (size_t)cr[k].idx * dp;
                    if (C->length != L) { same = 0; break; }
                    materialize(s, cs, dec, L, C->use_edits, m1);
                    if (memcmp(m0, m1, (size_t)L) != 0) same = 0;
                }
                if (same) { memcpy(outseq, m0, (size_t)L); corrected = 1; label = 2; }
            } else {
                materialize(s, aseq, dec, L, A->use_edits, outseq);
                corrected = 1; label = 1;
            }
        }
        fputc(r->fasta ? '>' : '@', fp);
        fputs(h, fp);
        if (o->quality_labels && (int64_t)i <= last) fprintf(fp, " care:q=%d", corrected ? label : 0);
        fputc('\n', fp);
        fwrite(outseq, 1, (size_t)L, fp);
        fputc('\n', fp);
        if (!r->fasta) { fputs("+\n", fp); fwrite(q, 1, strlen(q), fp); fputc('\n', fp); }
    }
    free(cr); free(dec); free(m0); free(m1); free(outseq);
    fclose(fp);
    return 0;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

int co_run(const char* const* infiles, int nfiles, const char* outfile, const co_opts* o, double* step2) {
    co_reads* r = co_reads_from_files(infiles, nfiles, o);
    if (!r) return -1;
    co_tables* tb = co_build_tables(r, o);
    const double t0 = now_s();
    co_results* res = co_correct(r, tb, o, 0, r->n, o->threads);
    const double t1 = now_s();
    if (step2) *step2 = t1 - t0;
    const int rc = co_write_output(r, res, o, outfile);
    co_results_free(res);
    co_tables_free(tb);
    co_reads_free(r);
    return rc;
}
