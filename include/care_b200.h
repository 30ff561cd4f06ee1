/*
 * care_b200.h -- C ABI of the B200 (sm_100a) read-correction library.
 *
 * This is the drop-in boundary for CARE's per-anchor correction path
 * (yanlifeng/CARE). Each entry point names the reference interface it
 * replaces. All functions return 0 on success and a negative
 * CARE_B200_E* code on failure; care_b200_last_error() returns a message.
 * No exception crosses this boundary. One context per host thread; calls on
 * one context are serial. The caller owns every host array it passes in;
 * the context owns all device memory and the result buffers it returns.
 */
#ifndef CARE_B200_H
#define CARE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CARE_B200_OK            0
#define CARE_B200_EINVAL       -1   /* invalid argument / option */
#define CARE_B200_ECUDA        -2   /* CUDA runtime error */
#define CARE_B200_ENOMEM       -3   /* device or host allocation failed */
#define CARE_B200_ESTATE       -4   /* call out of order (e.g. no reads uploaded) */
#define CARE_B200_EIO          -5   /* file read / write error */
#define CARE_B200_ELIMIT       -6   /* input beyond a documented limit */

/* The ProgramOptions fields read on the correction path
 * (include/options.hpp:36-123 of the reference; defaults :37-98). */
typedef struct care_b200_options {
    int   kmerlength;               /* -k, default 20 */
    int   num_maps;                 /* -h, default 48 (<= 48) */
    int   min_overlap;              /* --minalignmentoverlap, 30 */
    float max_error_rate;           /* --maxmismatchratio, 0.2 */
    float min_overlap_ratio;        /* --minalignmentoverlapratio, 0.30 */
    float estimated_errorrate;      /* --errorfactortuning, 0.06 */
    float estimated_coverage;       /* -c, mandatory */
    float m_coverage;               /* --coveragefactortuning, 0.6 */
    float paired_filter_threshold;  /* --pairedFilterThreshold, 0.06 */
    int   new_columns_to_correct;   /* --candidateCorrectionNewColumns, 15 */
    int   use_quality;              /* -q */
    int   quality_bits;             /* --qualityScoreBits: 1, 2 or 8 */
    int   exclude_ambiguous;        /* --excludeAmbiguous */
    int   correct_candidates;       /* --candidateCorrection */
    int   paired_end;               /* --pairmode PE */
    int   correction_type;          /* 0 classic consensus rule, 1 learned (MLP) */
    int   quality_labels;           /* --correctionQualityLabels */
    int   threads;                  /* host threads for STEP1/STEP3 helpers */
    int   device;                   /* CUDA device ordinal */
    int   batch_size;               /* anchors per device batch, 0 = automatic (as many as half of
                                       the free device memory holds, at least 2^20) */
    int   clf_min_coverage;         /* learned form: decision columns with a lower
                                       coverage keep the classic rule, default 3 */
} care_b200_options;

typedef struct care_b200_ctx care_b200_ctx;

/* Result view of the last correction call. Buffers are owned by the context
 * and stay valid until the next correction call or care_b200_destroy().
 * anchor_status bits: 1 = corrected, 2 = high quality (HQ) MSA,
 * 4 = store as edit list (the reference's useEdits, corrector.hpp:1648-1675).
 * Candidate corrections are in forward read orientation
 * (corrector.hpp:1679-1757). Sequences are max_length bytes per row, zero
 * past the read's length; rows of anchors that were not corrected are zero. */
typedef struct care_b200_results {
    uint32_t        first_anchor;
    uint32_t        num_anchors;
    int32_t         max_length;
    const uint8_t*  anchor_status;
    const int32_t*  anchor_num_edits;
    const char*     anchor_sequences;
    uint64_t        num_candidates;
    const uint32_t* cand_read_ids;
    const uint32_t* cand_anchor_ids;
    const int32_t*  cand_shifts;
    const uint8_t*  cand_use_edits;
    const char*     cand_sequences;
} care_b200_results;

void        care_b200_default_options(care_b200_options* opt);

/* Creates a context on opt->device. Replaces the CpuErrorCorrector
 * constructor (include/corrector.hpp:118-139): options, pitches and handles
 * are bound once; the read storage and minhasher follow by upload/build. */
int         care_b200_create(const care_b200_options* opt, care_b200_ctx** ctx);
int         care_b200_destroy(care_b200_ctx* ctx);
const char* care_b200_last_error(const care_b200_ctx* ctx);

/* Read-storage handle: replaces CpuReadStorage (include/cpureadstorage.hpp:
 * 11-84, gathers chunkedreadstorage.hpp:403-607). packed: num_reads rows of
 * pitch_ints uint32, 2-bit MSB-first (A=0,C=1,G=2,T=3, sequencehelpers.hpp:
 * 152-187); enc_quals: num_reads rows of qual_pitch_ints uint32 in the
 * reference's qualityScoreBits encoding (qualityscorecompression.hpp:90-119),
 * or NULL; ambiguous_ids: reads that contained non-ACGT bases. Data is
 * copied into HBM once. Read length limit: 256 bases, so pitch_ints is at
 * most 16 and qual_pitch_ints at most the words of 256 qualities (16, 8 or
 * 64 for 2-, 1- and 8-bit codes; CARE_B200_EINVAL otherwise). Re-uploading the same
 * number of reads keeps the tables (they index reads by id); a different
 * number drops them. */
int care_b200_upload_reads(care_b200_ctx* ctx, const uint32_t* packed, size_t pitch_ints,
                           const int32_t* lengths, const uint32_t* enc_quals,
                           size_t qual_pitch_ints, const uint32_t* ambiguous_ids,
                           size_t num_ambiguous, uint32_t num_reads);

/* Minhasher handle, host-built tables: replaces OrdinaryCpuMinhasher's
 * tables (ordinaryminhasher.hpp:98-221; content groupbykey.hpp:99-249).
 * For map m: keys[m][0..nkeys[m]) ascending, values of key i are
 * values[m][offsets[m][i] .. offsets[m][i+1]) ascending read ids. */
int care_b200_upload_tables(care_b200_ctx* ctx, int num_maps, const uint64_t* const* keys,
                            const uint32_t* const* offsets, const uint32_t* const* values,
                            const size_t* nkeys);

/* Builds the minhash tables from the uploaded reads: signatures on the GPU,
 * grouping with the reference's bucket rules (size < 2 or > threshold
 * cleared). Replaces constructCpuMinhasherFromReadStorage
 * (src/cpuminhasherconstruction.cpp:27-165). */
int care_b200_build_tables(care_b200_ctx* ctx);

/* Copies the device tables back in the upload_tables layout (for
 * inspection and tests). Arrays are owned by the context. */
int care_b200_get_table(care_b200_ctx* ctx, int map, const uint64_t** keys,
                        const uint32_t** offsets, const uint32_t** values, size_t* nkeys);

/* The hot path: corrects anchors [first_anchor, first_anchor+num_anchors).
 * Replaces CpuErrorCorrector::process / processMulti
 * (include/corrector.hpp:145-312, :325-513) over the correct_cpu loop
 * (src/correct_cpu.cpp:134-301). Paired-end ranges must be pair aligned
 * (even first and count, corrector.hpp:328). */
int care_b200_correct_range(care_b200_ctx* ctx, uint32_t first_anchor, uint32_t num_anchors,
                            care_b200_results* results);

/* Same work without the device->host copy of results: the results stay in
 * HBM (used to time the device pipeline alone). */
int care_b200_correct_range_device(care_b200_ctx* ctx, uint32_t first_anchor,
                                   uint32_t num_anchors);

/* Serialises the results as the reference's EncodedTempCorrectedSequence
 * byte records (correctedsequence.hpp:148-340: readId u32, flags u32 with
 * bit31 hq, bit30 useEdits, bit29 type, low 29 bits payload size, payload),
 * applying the save filter of src/correct_cpu.cpp:255-273. With out == NULL
 * only *needed is set. */
int care_b200_serialize_results(care_b200_ctx* ctx, const care_b200_results* results,
                                uint8_t* out, size_t capacity, size_t* needed);

/* ---- whole-file driver (STEP1 + STEP2 + STEP3 of care-cpu,
 *      src/dispatch_care_correct_cpu.cpp:51-251) ---- */

/* Parses FASTQ/FASTA (one file, or two files of mates for PE), applies the
 * reference's read preprocessing (chunkedreadstorageconstruction.hpp:67-92)
 * and uploads the read storage. */
int care_b200_load_reads_from_files(care_b200_ctx* ctx, const char* const* files, int num_files);

/* The same storage, parsed and encoded on the device (STEP1's parse and
 * encode, include/chunkedreadstorageconstruction.hpp:29-400 and
 * include/qualityscorecompression.hpp:90-119): the files' bytes are copied
 * to the device once, line ends and records are found by device scans, the
 * N-rotation counter (restarting every 65,536-read parser batch) by a scan of
 * each read's ambiguous characters, and every read is encoded by one warp.
 * For records in strict 4-line FASTQ or 2-line FASTA layout (a missing last
 * line end and CRLF line ends included); any other layout returns
 * CARE_B200_EINVAL with the storage unchanged, and
 * care_b200_load_reads_from_files reads it. The output records are written
 * from the same bytes (care_b200_write_output). */
int care_b200_load_reads_from_files_device(care_b200_ctx* ctx, const char* const* files, int num_files);

/* Read-storage handle, binary file: uploads the read storage that care-cpu
 * saved with --save-preprocessedreads-to (ChunkedReadStorage::loadFromFile,
 * include/chunkedreadstorage.hpp:160-243), in place of parsing FASTQ. As in the
 * reference, a file whose quality bits differ from the options, or without
 * qualities when the options use them, is rejected; qualities the options do
 * not use are skipped. The file holds no input records: output records from
 * an earlier care_b200_load_reads_from_files of the same reads stay in use for
 * care_b200_write_output (care-cpu, too, writes its output from the input
 * files); otherwise use care_b200_serialize_results. */
int care_b200_load_preprocessed_reads(care_b200_ctx* ctx, const char* path);

/* Writes the uploaded read storage in the same layout
 * (ChunkedReadStorage::saveToFile, include/chunkedreadstorage.hpp:246-398);
 * ambiguous read ids in ascending order. */
int care_b200_save_preprocessed_reads(care_b200_ctx* ctx, const char* path);

/* Minhasher handle, binary file: uploads the tables care-cpu saved with
 * --save-hashtables-to (OrdinaryCpuMinhasher::loadFromStream,
 * include/ordinaryminhasher.hpp:318-339), in place of care_b200_build_tables.
 * As in the reference, at most num_maps maps are loaded and the file's k-mer
 * length and per-map result threshold are used. The read storage must be the
 * one the tables were built from (read ids are checked against its size). */
int care_b200_load_hashtables(care_b200_ctx* ctx, const char* path);

/* Writes the tables in the same layout, byte for byte what care-cpu writes
 * for the same tables (OrdinaryCpuMinhasher::writeToStream,
 * include/ordinaryminhasher.hpp:303-316; load factor 0.8). */
int care_b200_save_hashtables(care_b200_ctx* ctx, const char* path);

/* Merges all corrections of the last full-range call with the input reads
 * and writes the output file (correctionresultoutput.cpp:30-440, 730-1020). */
int care_b200_write_output(care_b200_ctx* ctx, const char* outfile);

/* Statistics of the last correction call: device milliseconds of the
 * pipeline and per-stage kernel times: stage_ms[0] candidate lookup (table
 * queries of the anchors' resident signatures), [1] alignment, [2] MSA and
 * correction, [3] the learned decision. stage_ms[4], when asked for, is the
 * last minhash-signature pass over the read storage (run once per uploaded
 * or loaded storage, not by the correction calls). */
int care_b200_last_timing(const care_b200_ctx* ctx, float* total_ms, float* stage_ms, int nstages);

/* Counters of the last correction call: stats[0] anchors, stats[1]
 * (anchor, candidate) pairs aligned, stats[2] candidate corrections,
 * stats[3] un-pruned 32-bit word compares of the alignment scans run (both
 * orientations, every scanned shift; a mirrored pair's shared scans count
 * once: the alignment stage's roofline work),
 * stats[4] bases added to MSA column sums (anchor and candidates, every
 * build including refinement rebuilds: the MSA stage's compute work),
 * stats[5] device batches the range was split into, stats[6] kernels of
 * this library launched (every batch and every arena-growth attempt),
 * stats[7] anchors whose candidate lists took the second, full-set pass,
 * stats[8] 32-bit word compares the alignment scans actually ran after their
 * early exits (counted only while care_b200_count_word_compares is on, else 0),
 * stats[9] bases added to MSA column sums by refinement rebuilds (the builds
 * after an anchor's first; included in stats[4]), stats[10] anchors whose
 * MSA was rebuilt at least once (refineMSA, include/corrector.hpp:1307-1421). */
int care_b200_last_stats(const care_b200_ctx* ctx, uint64_t* stats, int nstats);

/* on = 1: the following correction calls run the alignment's statistics form,
 * which also counts the word compares its scans run (stats[8]; the reference's
 * early exit, src/cpu_alignment.cpp:82-98, is what makes this count smaller than
 * stats[3]). Slower; results unchanged. on = 0 (default) turns it off. */
int care_b200_count_word_compares(care_b200_ctx* ctx, int on);

/* ---- correction without allocation ---- */

/* Device-resident read storage owned by the caller (layout of
 * care_b200_upload_reads: 2-bit rows, encoded quality rows, lengths, and
 * one byte per read, nonzero for reads that contained non-ACGT bases). */
typedef struct care_b200_device_reads {
    const uint32_t* packed;
    size_t          pitch_ints;
    const int32_t*  lengths;
    const uint32_t* quals;            /* NULL when qualities are not used */
    size_t          qual_pitch_ints;
    const uint8_t*  ambiguous;
    uint32_t        num_reads;
    int             max_length;       /* longest read of the storage (<= 256) */
} care_b200_device_reads;

/* Device-resident minhash tables owned by the caller, in the layout this
 * library builds: per map a descriptor {uint64 slot_base; uint64 value_base;
 * uint32 mask; uint32 pad} (24 bytes), an open-addressing slot array of
 * {uint64 key; uint32 offset; uint32 count} (16 bytes; count 0 = empty;
 * capacity mask+1 a power of two; a key starts probing at
 * MurmurHash3-fmix64(key) & mask and moves to the next slot), and one value
 * array of read ids (the key's ids at value_base + offset, ascending; every
 * id below the storage's num_reads). */
typedef struct care_b200_device_tables {
    int             num_maps;
    const void*     descs;
    const void*     slots;
    const uint32_t* values;
    int             threshold;        /* per-map result threshold of these tables
                                         (care_b200_result_threshold); 0: derived
                                         from opt->estimated_coverage */
} care_b200_device_tables;

#define CARE_B200_NOALLOC_MAX_ANCHORS 16384
#define CARE_B200_NOALLOC_MAX_PAIRS   1048576

/* Anchor correction of [first_anchor, first_anchor+num_anchors) that
 * allocates nothing, for callers that cannot call cudaMalloc (buffers laid
 * out by a host framework's own pool or mapped from another process, or code
 * that must not change the device's memory map while it runs). No
 * counterpart in the reference. Inputs and outputs are device pointers the
 * caller owns: status (1 byte per anchor, same bits as care_b200_results),
 * num_edits (int32 per anchor) and sequences (max_length bytes per anchor;
 * rows of uncorrected anchors are zero). Candidate correction is not
 * available here (opt->correct_candidates must be 0). Work runs on `stream`
 * (a cudaStream_t, NULL for the default stream) and the call returns when it
 * has finished.
 * Working memory is one device array compiled into the library (about 32 MB):
 * at most CARE_B200_NOALLOC_MAX_ANCHORS anchors and
 * CARE_B200_NOALLOC_MAX_PAIRS (anchor, candidate) pairs per call; larger
 * requests return CARE_B200_ELIMIT. CUDA places a module's device arrays
 * when the module is first used, so the array is reserved by the first call
 * on each device (which also looks up its address and loads constants) and
 * then held until the process exits: make that first call before the
 * caller's own pool takes the device's memory, and before any stream
 * capture; later calls leave the device's free memory unchanged. Every read
 * length must lie in [0, max_length] (checked on the device first:
 * CARE_B200_EINVAL otherwise), and with qualities qual_pitch_ints must hold
 * max_length * quality_bits bits. All calls share the array: calls that
 * overlap on the GPU (from several threads or streams) race and must be
 * serialised by the caller.
 * Returns 0 or a CARE_B200_E* code. */
int care_b200_correct_range_noalloc(const care_b200_options* opt, const care_b200_device_reads* reads,
                                    const care_b200_device_tables* tables, uint32_t first_anchor,
                                    uint32_t num_anchors, uint8_t* status, int32_t* num_edits,
                                    char* sequences, void* stream);

/* ---- learned decision (correction_type 1) ----
 *
 * The reference's classifier hook, correctAnchorClf (corrector.hpp:1448-1472)
 * with ClfAgent::decide_anchor (classification.hpp:123-133), asks for every
 * anchor position of a non-HQ MSA whose base differs from the consensus
 * whether the consensus base is written. Here a 24 -> 64 -> 64 -> 1 MLP with
 * GELU answers (logit > 0: write the consensus); positions whose column
 * coverage is below clf_min_coverage keep the classic rule. The reference
 * serves the hook with a random forest read from a file (forest.hpp:217-226);
 * the network, its training kernels and the feature rows are this library's
 * own.
 *
 * Parameter vector (float32, CARE_B200_MLP_FLOATS): W1[64][24] b1[64]
 * W2[64][64] b2[64] w3[64] b3 (the CARE_B200_MLP_PARAMS trained values),
 * then the input normalisation mean[24] inv_std[24]. Weights and hidden
 * activations enter the tensor-core GEMMs as bfloat16 with FP32
 * accumulation. */
#define CARE_B200_MLP_FEATURES 24
#define CARE_B200_MLP_HIDDEN   64
#define CARE_B200_MLP_PARAMS   5825
#define CARE_B200_MLP_FLOATS   5873

/* Decision-column rows of the last care_b200_collect_features() call, owned
 * by the context. meta = position | orig << 16 | cons << 18 (2-bit base
 * codes A=0 C=1 G=2 T=3); logits only when the network decided. Row order is
 * unspecified. */
typedef struct care_b200_features {
    uint64_t        count;
    const float*    x;                /* count * 24 */
    const uint32_t* read_ids;
    const uint32_t* meta;
    const float*    logits;           /* NULL under correction_type 0 */
} care_b200_features;

/* Parameters used by correction_type 1 (copied). */
int care_b200_set_mlp(care_b200_ctx* ctx, const float* params);

/* care_b200_correct_range() that also returns the decision-column rows:
 * under correction_type 0 the rows the classic rule passed over (training
 * data), under correction_type 1 the rows the network decided. */
int care_b200_collect_features(care_b200_ctx* ctx, uint32_t first_anchor, uint32_t num_anchors,
                               care_b200_results* results, care_b200_features* features);

/* Training and batched inference of the network on one device. */
typedef struct care_b200_mlp care_b200_mlp;

typedef struct care_b200_mlp_train_options {
    int      epochs;
    int      batch;                   /* rows per Adam step, e.g. 65536 */
    double   lr, beta1, beta2, eps;   /* Adam: 1e-3, 0.9, 0.999, 1e-8 */
    uint64_t seed;                    /* row shuffling */
} care_b200_mlp_train_options;

void        care_b200_mlp_default_train_options(care_b200_mlp_train_options* o);
int         care_b200_mlp_create(int device, care_b200_mlp** out);
int         care_b200_mlp_destroy(care_b200_mlp* m);
const char* care_b200_mlp_last_error(const care_b200_mlp* m);
/* parameters in and out (CARE_B200_MLP_FLOATS); setting resets Adam */
int care_b200_mlp_set_params(care_b200_mlp* m, const float* params);
int care_b200_mlp_get_params(care_b200_mlp* m, float* params);
/* uniform fan-in initialisation of the trained values (seeded) */
int care_b200_mlp_init(care_b200_mlp* m, uint64_t seed);
/* training rows made resident on the device (labels 0 or 1; weights scale
 * each row's loss, NULL = 1); with set_normalisation the mean and 1/std of
 * each feature are taken from them */
int care_b200_mlp_set_data(care_b200_mlp* m, const float* x, const float* labels, const float* weights,
                           uint64_t n, int set_normalisation);
/* Adam over the resident rows, shuffled each epoch, the whole run replayed as
 * one CUDA graph; losses (mean BCE per step) are written when non-NULL */
int care_b200_mlp_train(care_b200_mlp* m, const care_b200_mlp_train_options* o, float* losses,
                        uint64_t loss_capacity, uint64_t* num_steps);
/* gradient (CARE_B200_MLP_PARAMS) and loss of host rows: sum over rows of
 * weight * BCE(logit, label), divided by the row count (weights NULL = 1) */
int care_b200_mlp_gradient(care_b200_mlp* m, const float* x, const float* labels, const float* weights,
                           uint64_t n, float* grad, float* loss);
/* one Adam step on host rows */
int care_b200_mlp_train_step(care_b200_mlp* m, const float* x, const float* labels, const float* weights,
                             uint64_t n, const care_b200_mlp_train_options* o, float* loss);
/* logits of host rows */
int care_b200_mlp_forward(care_b200_mlp* m, const float* x, uint64_t n, float* logits);

/* ---- launch mapping (tuning) ----
 *
 * How the batch's work is mapped onto the GPU; the results do not depend on
 * it (every variant is byte-identical). care_b200.autotune measures the
 * variants on a sample of a workload and commits the fastest per workload. */
typedef struct care_b200_tuning {
    int msa_order;     /* 1: anchors in longest-processing-time order (most candidates first) */
    int msa_queue;     /* 1: persistent MSA CTAs pulling anchors from a device work queue */
    int msa_warps;     /* warps per anchor in the MSA stage: 4 or 8 */
    int align_block;   /* threads per CTA of the alignment stage: 128 or 256 */
    int pair_order;    /* 1: alignment pairs packed by candidate length within each anchor */
    int graph;         /* 1: each batch's launches replayed as one CUDA graph */
    int pair_mirror;   /* 1: pairs (a, c) and (c, a) of equal-length anchors of one batch share
                          their scans (one scan answers both forward alignments) */
    int cand_set_log2; /* 6..14: de-duplication set of the main candidate pass, 2^x entries;
                          anchors with more than 2^(x-1) unique candidates take a second pass
                          with a set for every retrieved id (default 10) */
    int align_warp;    /* 1: a warp per alignment work item, its lanes taking the shifts of
                          each group of 32 (the scan's first minimal shift found by warp
                          reductions); 0: a thread per work item */
    int align_classes; /* 1: the batch's pairs partitioned by the plane width their longer read
                          needs (4/5/6/8 words of 32 bases), one alignment launch per class
                          (no effect with pair_mirror) */
} care_b200_tuning;

int care_b200_default_tuning(care_b200_tuning* t);
int care_b200_set_tuning(care_b200_ctx* ctx, const care_b200_tuning* t);
int care_b200_get_tuning(const care_b200_ctx* ctx, care_b200_tuning* t);

/* Read-storage facts after upload. */
uint32_t care_b200_num_reads(const care_b200_ctx* ctx);
int      care_b200_max_length(const care_b200_ctx* ctx);
int      care_b200_num_maps(const care_b200_ctx* ctx);
/* Per-map result threshold of the context's tables: buckets with more read
 * ids are dropped at query time (OrdinaryCpuMinhasher::queryMap,
 * include/ordinaryminhasher.hpp:437-449). Derived from the coverage
 * (calculateResultsPerMapThreshold, include/minhasherlimit.hpp:9-15) unless
 * tables were loaded from a file, whose own threshold is then used. */
int      care_b200_result_threshold(const care_b200_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
