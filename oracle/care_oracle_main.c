/*
 * care_oracle_main.c -- command line of the CPU restatement (test
 * infrastructure only). Accepts the subset of care-cpu's options that the
 * correction path reads (src/options.cpp:54-383, src/main_correct_cpu.cpp)
 * and prints care-cpu's throughput line
 * (src/dispatch_care_correct_cpu.cpp:168).
 */
#define _GNU_SOURCE
#include "care_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

static int is_true(const char* v) { return !v || strcmp(v, "true") == 0 || strcmp(v, "1") == 0; }

int main(int argc, char** argv) {
    co_opts o;
    co_default_opts(&o);
    const char* in[2] = {0, 0};
    int nin = 0;
    const char* outdir = ".";
    const char* outname = NULL;
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        const char* v = i + 1 < argc ? argv[i + 1] : NULL;
#define ARG(s) (strcmp(a, s) == 0)
        if (ARG("-i") || ARG("--inputfiles")) {
            char* list = strdup(v); i++;
            for (char* tok = strtok(list, ","); tok && nin < 2; tok = strtok(NULL, ",")) in[nin++] = tok;
        } else if (ARG("-d") || ARG("--outdir")) { outdir = v; i++; }
        else if (ARG("-o") || ARG("--outputfilenames")) { outname = v; i++; }
        else if (ARG("-c") || ARG("--coverage")) { o.estimated_coverage = (float)atof(v); i++; }
        else if (ARG("-k") || ARG("--kmerlength")) { o.kmerlength = atoi(v); i++; }
        else if (ARG("-h") || ARG("--hashmaps")) { o.num_maps = atoi(v); i++; }
        else if (ARG("-t") || ARG("--threads")) { o.threads = atoi(v); i++; }
        else if (ARG("--pairmode")) { o.paired_end = (strcmp(v, "PE") == 0 || strcmp(v, "pe") == 0); i++; }
        else if (ARG("-q") || ARG("--useQualityScores")) { o.use_quality = 1; }
        else if (ARG("--qualityScoreBits")) { o.quality_bits = atoi(v); i++; }
        else if (ARG("--excludeAmbiguous")) { o.exclude_ambiguous = 1; }
        else if (ARG("--candidateCorrection")) { o.correct_candidates = 1; }
        else if (ARG("--correctionQualityLabels")) { o.quality_labels = 1; }
        else if (ARG("--minalignmentoverlap")) { o.min_overlap = atoi(v); i++; }
        else if (ARG("--maxmismatchratio")) { o.max_error_rate = (float)atof(v); i++; }
        else if (ARG("--minalignmentoverlapratio")) { o.min_overlap_ratio = (float)atof(v); i++; }
        else if (ARG("--errorfactortuning")) { o.estimated_errorrate = (float)atof(v); i++; }
        else if (ARG("--coveragefactortuning")) { o.m_coverage = (float)atof(v); i++; }
        else if (ARG("--pairedFilterThreshold")) { o.paired_filter_threshold = (float)atof(v); i++; }
        else if (ARG("--candidateCorrectionNewColumns")) { o.new_columns_to_correct = atoi(v); i++; }
        else { fprintf(stderr, "care-oracle: unknown option %s\n", a); return 1; }
#undef ARG
        (void)is_true;
    }
    if (!nin || !outname) {
        fprintf(stderr, "usage: care-oracle -i reads.fq -d outdir -o out.fq -c cov --pairmode SE|PE [options]\n");
        return 1;
    }
    mkdir(outdir, 0755);
    char path[4096];
    snprintf(path, sizeof(path), "%s/%s", outdir, outname);
    double s2 = 0.0;
    co_reads* probe = NULL;
    (void)probe;
    const int rc = co_run(in, nin, path, &o, &s2);
    if (rc != 0) { fprintf(stderr, "care-oracle: failed (%d)\n", rc); return 1; }
    printf("STEP2 seconds: %.6f\n", s2);
    return 0;
}
