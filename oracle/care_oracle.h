/*
 * care_oracle.h -- CPU restatement of CARE's per-anchor correction path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the parity tests, smoke()
 * and bench.py's CPU-baseline leg compare the CUDA product against. The
 * product (care_b200/) never links, loads or calls it.
 *
 * Every function restates one piece of the reference (yanlifeng/CARE)
 * and cites the file:line it follows. Parity of this restatement is pinned
 * against the reference's own care-cpu binary, compiled from its sources
 * by oracle/Makefile into oracle/_ref/care-cpu (tests/test_oracle_pin.py
 * and the golden fixtures under tests/golden/).
 */
#ifndef CARE_ORACLE_H
#define CARE_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The ProgramOptions fields on the correction path (include/options.hpp:36-98). */
typedef struct {
    int   kmerlength;               /* -k, default 20 */
    int   num_maps;                 /* -h, default 48 */
    int   min_overlap;              /* --minalignmentoverlap, 30 */
    float max_error_rate;           /* --maxmismatchratio, 0.2 */
    float min_overlap_ratio;        /* --minalignmentoverlapratio, 0.30 */
    float estimated_errorrate;      /* --errorfactortuning, 0.06 */
    float estimated_coverage;       /* -c */
    float m_coverage;               /* --coveragefactortuning, 0.6 */
    float paired_filter_threshold;  /* --pairedFilterThreshold, 0.06 */
    int   new_columns_to_correct;   /* --candidateCorrectionNewColumns, 15 */
    int   use_quality;              /* -q */
    int   quality_bits;             /* --qualityScoreBits, 8 */
    int   exclude_ambiguous;        /* --excludeAmbiguous */
    int   correct_candidates;       /* --candidateCorrection */
    int   paired_end;               /* --pairmode PE */
    int   threads;                  /* -t */
    int   quality_labels;           /* --correctionQualityLabels */
    /* classifier hook (correctAnchorClf, corrector.hpp:1448-1472): 0 = the
     * plain rule only; 1 = plain rule, decision columns reported as feature
     * rows; 2 = the MLP decides each decision column (plain rule below
     * clf_min_coverage) */
    int   clf_mode;
    int   clf_min_coverage;
    const float* mlp;               /* CO_MLP_FLOATS values, clf_mode 2 */
} co_opts;

/* ---- learned decision: features and the MLP ---- */
#define CO_NFEAT 24
#define CO_HIDDEN 64
/* parameter vector: W1[64][24] b1[64] W2[64][64] b2[64] w3[64] b3, then the
 * input normalisation mean[24] inv_std[24] */
#define CO_MLP_W1 0
#define CO_MLP_B1 1536
#define CO_MLP_W2 1600
#define CO_MLP_B2 5696
#define CO_MLP_W3 5760
#define CO_MLP_B3 5824
#define CO_MLP_NPARAM 5825
#define CO_MLP_MEAN 5825
#define CO_MLP_ISTD 5849
#define CO_MLP_FLOATS 5873

/* One decision column: an anchor position of a non-HQ MSA whose original
 * base differs from the consensus (orig/cons are 2-bit codes). */
typedef struct {
    uint32_t read_id;
    int16_t  pos;
    uint8_t  orig, cons;
    float    logit;                 /* clf_mode 2 only */
    float    x[CO_NFEAT];
} co_feature;

void co_default_opts(co_opts* o);

/* In-memory read storage (the content of ChunkedReadStorage after
 * construction, include/chunkedreadstorageconstruction.hpp:29-485). */
typedef struct {
    uint32_t  n;
    int       min_len, max_len;
    int       seq_pitch;      /* uint32 per read, ceil(max_len/16) */
    int       qual_pitch;     /* uint32 per read, ceil(max_len*bits/32) */
    int       quality_bits;
    int       has_quality;
    uint32_t* seq;            /* n * seq_pitch, 2-bit MSB-first, zero padded */
    uint32_t* qual;           /* n * qual_pitch, encoded qualities */
    int32_t*  len;
    uint8_t*  ambig;          /* 1 if the input read had a non-ACGTacgt base */
    /* original records, kept for output construction */
    char*     text;           /* concatenated header\0seq\0qual\0 */
    size_t*   rec_off;        /* n offsets into text */
    int       fasta;
} co_reads;

/* One minhash table: keys sorted ascending, values grouped per key and
 * sorted ascending (include/groupbykey.hpp:99-249). */
typedef struct {
    uint64_t* keys;
    uint32_t* offsets;        /* nkeys + 1 */
    uint32_t* values;
    size_t    nkeys;
} co_table;

typedef struct {
    int       num_maps;
    int       k;
    int       threshold;      /* resultsPerMapThreshold */
    co_table* t;
} co_tables;

/* Per-anchor outcome.  status: 0 = no anchor correction, 1 = corrected. */
typedef struct {
    uint8_t status;
    uint8_t hq;
    uint8_t use_edits;
    uint8_t pad;
    int32_t num_edits;
} co_anchor_result;

typedef struct {
    uint32_t read_id;         /* corrected candidate read */
    uint32_t anchor_id;       /* anchor whose MSA produced it */
    int32_t  shift;
    int32_t  length;
    uint8_t  use_edits;
    uint8_t  pad[3];
} co_cand_result;

typedef struct {
    uint32_t          first, count;
    int               max_len;
    co_anchor_result* anchors;     /* count */
    char*             anchor_seq;  /* count * max_len corrected anchor */
    /* candidate corrections, in anchor order then candidate order */
    co_cand_result*   cands;
    char*             cand_seq;    /* num_cands * max_len, forward orientation */
    size_t            num_cands, cap_cands;
    /* decision columns (clf_mode 1 and 2), in anchor then position order */
    co_feature*       feats;
    size_t            num_feats, cap_feats;
} co_results;

/* ---- end-to-end (STEP1 + STEP2 + STEP3 of care-cpu) ---- */
co_reads*  co_reads_from_files(const char* const* files, int nfiles, const co_opts* o);
void       co_reads_free(co_reads* r);
co_tables* co_build_tables(const co_reads* r, const co_opts* o);
void       co_tables_free(co_tables* t);
co_results* co_correct(const co_reads* r, const co_tables* t, const co_opts* o,
                       uint32_t first, uint32_t count, int threads);
void       co_results_free(co_results* res);
int        co_write_output(const co_reads* r, const co_results* res, const co_opts* o,
                           const char* outfile);
int        co_run(const char* const* infiles, int nfiles, const char* outfile,
                  const co_opts* o, double* step2_seconds);

/* ---- stage functions, exposed for known-answer tests ---- */
void     co_encode_2bit(const char* s, int len, uint32_t* out);
void     co_decode_2bit(const uint32_t* enc, int len, char* out);
void     co_revcomp_2bit(const uint32_t* in, int len, uint32_t* out);
void     co_to_hilo(const uint32_t* in, int len, uint32_t* out);
uint64_t co_murmur64(uint64_t x);
void     co_signature(const uint32_t* seq, int len, int k, int num_maps, uint64_t* out);
int      co_threshold(float coverage);
void     co_encode_quality(const char* q, int len, int bits, uint32_t* out);
void     co_decode_quality(const uint32_t* enc, int len, int bits, char* out);
void     co_quality_weights(float* out256);
float    co_bf16_round(float x);
float    co_mlp_logit(const float* params, const float* x);

typedef struct {
    int score, overlap, shift, nops, valid;
} co_align;

void co_shd(const uint32_t* anchor2bit, int la, const uint32_t* cand2bit, int lc,
            int min_overlap, float max_error_rate, float min_overlap_ratio, co_align* out);
int  co_orientation(const co_align* fwd, const co_align* rc, int la, int lc,
                    float min_overlap_ratio, int min_overlap, float estimated_errorrate);
void co_pair_flags(const uint32_t* l1, int n1, const uint32_t* l2, int n2,
                   uint8_t* f1, uint8_t* f2);

/* Trace of one anchor's candidate set at the end of the path (after the
 * alignment filters and MSA refinement), for stage-level parity checks. */
typedef struct {
    int      n_initial;       /* after minhash query, dedup, self removal */
    int      n_after_flag;    /* after orientation filter */
    int      n_after_ratio;   /* after mismatch-ratio filter */
    int      n_final;         /* after refinement */
    int      n_columns;
    int      anchor_col_begin;
} co_trace;

int co_trace_anchor(const co_reads* r, const co_tables* t, const co_opts* o,
                    uint32_t anchor, co_trace* tr,
                    uint32_t* ids, int* shifts, int* orient, float* weights, int cap,
                    uint32_t* initial_ids, int initial_cap);

#ifdef __cplusplus
}
#endif
#endif
