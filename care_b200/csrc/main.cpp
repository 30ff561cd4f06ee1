// care-b200: the correction pipeline with care-cpu's command line
// (src/main_correct_cpu.cpp:60-152, options src/options.cpp:54-383 and
// :700-913 of the reference). STEP1 builds the read storage and minhash
// tables, STEP2 runs the device path, STEP3 writes the corrected file.
#include "../../include/care_b200.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void usage() {
    std::puts(
        "care-b200 -i reads.fq [-i mates.fq] -d outdir -o out.fq -c coverage --pairmode SE|PE [options]\n"
        "  -k,--kmerlength N            -h,--hashmaps N          -t,--threads N\n"
        "  -q,--useQualityScores        --qualityScoreBits 1|2|8 --excludeAmbiguous\n"
        "  --candidateCorrection        --candidateCorrectionNewColumns N\n"
        "  --minalignmentoverlap N      --maxmismatchratio F     --minalignmentoverlapratio F\n"
        "  --errorfactortuning F        --coveragefactortuning F --pairedFilterThreshold F\n"
        "  --correctionQualityLabels    --batchsize N            -g,--gpu N\n"
        "  --correctionType 0|1 (1: learned decision)  --ml-mlpfile FILE  --clfMinCoverage N\n"
        "  --save-preprocessedreads-to FILE  --load-preprocessedreads-from FILE\n"
        "  --save-hashtables-to FILE         --load-hashtables-from FILE");
}

bool flag_value(int& i, int argc, char** argv) {
    // implicit-true boolean (cxxopts implicit_value("true")), optional explicit value
    if (i + 1 < argc && (std::strcmp(argv[i + 1], "true") == 0 || std::strcmp(argv[i + 1], "false") == 0)) {
        return std::strcmp(argv[++i], "true") == 0;
    }
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    care_b200_options o;
    care_b200_default_options(&o);
    std::vector<std::string> inputs;
    std::string outdir, outname, mlpfile, save_reads, load_reads, save_tables, load_tables;
    bool haveCov = false, havePair = false;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto val = [&]() -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(1); }
            return argv[++i];
        };
        if (a == "-i" || a == "--inputfiles") {
            std::string v = val();
            size_t p = 0;
            while (p <= v.size()) {
                const size_t q = v.find(',', p);
                inputs.push_back(v.substr(p, q == std::string::npos ? std::string::npos : q - p));
                if (q == std::string::npos) break;
                p = q + 1;
            }
        } else if (a == "-d" || a == "--outdir") outdir = val();
        else if (a == "-o" || a == "--outputfilenames") outname = val();
        else if (a == "-c" || a == "--coverage") { o.estimated_coverage = (float)std::atof(val()); haveCov = true; }
        else if (a == "-k" || a == "--kmerlength") o.kmerlength = std::atoi(val());
        else if (a == "-h" || a == "--hashmaps") o.num_maps = std::atoi(val());
        else if (a == "-t" || a == "--threads") o.threads = std::atoi(val());
        else if (a == "-g" || a == "--gpu") o.device = std::atoi(val());
        else if (a == "--pairmode") {
            const std::string v = val();
            havePair = true;
            if (v == "PE" || v == "pe") o.paired_end = 1;
            else if (v == "SE" || v == "se") o.paired_end = 0;
            else { std::fprintf(stderr, "invalid pairmode %s\n", v.c_str()); return 1; }
        } else if (a == "-q" || a == "--useQualityScores") o.use_quality = flag_value(i, argc, argv);
        else if (a == "--qualityScoreBits") o.quality_bits = std::atoi(val());
        else if (a == "--excludeAmbiguous") o.exclude_ambiguous = flag_value(i, argc, argv);
        else if (a == "--candidateCorrection") o.correct_candidates = flag_value(i, argc, argv);
        else if (a == "--correctionQualityLabels") o.quality_labels = flag_value(i, argc, argv);
        else if (a == "--candidateCorrectionNewColumns") o.new_columns_to_correct = std::atoi(val());
        else if (a == "--minalignmentoverlap") o.min_overlap = std::atoi(val());
        else if (a == "--maxmismatchratio") o.max_error_rate = (float)std::atof(val());
        else if (a == "--minalignmentoverlapratio") o.min_overlap_ratio = (float)std::atof(val());
        else if (a == "--errorfactortuning") o.estimated_errorrate = (float)std::atof(val());
        else if (a == "--coveragefactortuning") o.m_coverage = (float)std::atof(val());
        else if (a == "--pairedFilterThreshold") o.paired_filter_threshold = (float)std::atof(val());
        else if (a == "--batchsize") o.batch_size = std::atoi(val());
        else if (a == "--correctionType") o.correction_type = std::atoi(val()) == 1 ? 1 : 0;
        else if (a == "--ml-mlpfile") mlpfile = val();
        else if (a == "--clfMinCoverage") o.clf_min_coverage = std::atoi(val());
        else if (a == "--save-preprocessedreads-to") save_reads = val();
        else if (a == "--load-preprocessedreads-from") load_reads = val();
        else if (a == "--save-hashtables-to") save_tables = val();
        else if (a == "--load-hashtables-from") load_tables = val();
        else if (a == "--help") { usage(); return 0; }
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); usage(); return 1; }
    }
    // mandatory arguments (src/main_correct_cpu.cpp:32-48)
    if (inputs.empty() || outdir.empty() || outname.empty() || !haveCov || !havePair) { usage(); return 0; }
    mkdir(outdir.c_str(), 0755);
    const std::string outpath = outdir + "/" + outname;

    care_b200_ctx* ctx = nullptr;
    int rc = care_b200_create(&o, &ctx);
    if (rc) { std::fprintf(stderr, "care-b200: create failed (%d)%s%s\n", rc, ctx ? ": " : "", ctx ? care_b200_last_error(ctx) : ""); return 1; }
    auto die = [&](const char* what) {
        std::fprintf(stderr, "care-b200: %s: %s\n", what, care_b200_last_error(ctx));
        care_b200_destroy(ctx);
        return 1;
    };
    if (o.correction_type == 1) {
        // network parameters: CARE_B200_MLP_FLOATS little-endian float32 values
        std::vector<float> params(CARE_B200_MLP_FLOATS);
        FILE* f = mlpfile.empty() ? nullptr : std::fopen(mlpfile.c_str(), "rb");
        const bool ok = f && std::fread(params.data(), 4, params.size(), f) == params.size();
        if (f) std::fclose(f);
        if (!ok) {
            std::fprintf(stderr, "care-b200: --correctionType 1 needs --ml-mlpfile with %d float32 values\n", CARE_B200_MLP_FLOATS);
            care_b200_destroy(ctx);
            return 1;
        }
        if (care_b200_set_mlp(ctx, params.data())) return die("loading the network");
    }
    std::printf("STEP 1: Database construction\n");
    const double t0 = now();
    std::vector<const char*> fp;
    for (auto& s : inputs) fp.push_back(s.c_str());
    if (care_b200_load_reads_from_files(ctx, fp.data(), (int)fp.size())) return die("reading input");
    // as care-cpu: the read storage from the saved file, the output records
    // from the input files (constructChunkedReadStorageFromFiles,
    // include/chunkedreadstorageconstruction.hpp:35-42)
    if (!load_reads.empty() && care_b200_load_preprocessed_reads(ctx, load_reads.c_str()))
        return die("loading the saved read storage");
    if (!save_reads.empty()) {
        std::printf("Saving reads to file %s\n", save_reads.c_str());
        if (care_b200_save_preprocessed_reads(ctx, save_reads.c_str())) return die("saving the read storage");
    }
    if (!load_tables.empty()) {
        if (care_b200_load_hashtables(ctx, load_tables.c_str())) return die("loading the saved hash tables");
    } else if (care_b200_build_tables(ctx)) {
        return die("building hash tables");
    }
    if (!save_tables.empty()) {
        std::printf("Saving minhasher to file %s\n", save_tables.c_str());
        if (care_b200_save_hashtables(ctx, save_tables.c_str())) return die("saving the hash tables");
    }
    const double t1 = now();
    std::printf("Total number of reads: %u\nMaximum sequence length: %d\nUsing %d maps\n",
                care_b200_num_reads(ctx), care_b200_max_length(ctx), care_b200_num_maps(ctx));
    std::printf("STEP1: %.3f s\nSTEP 2: Error correction\n", t1 - t0);
    care_b200_results res;
    const uint32_t n = care_b200_num_reads(ctx);
    if (care_b200_correct_range(ctx, 0, n, &res)) return die("correction");
    const double t2 = now();
    std::printf("STEP2: %.3f s\n", t2 - t1);
    std::printf("Correction throughput : ~%.1f reads/second.\n", n / (t2 - t1));
    std::printf("STEP 3: Constructing output file(s)\n");
    if (care_b200_write_output(ctx, outpath.c_str())) return die("writing output");
    const double t3 = now();
    std::printf("STEP3: %.3f s\nConstruction of output file(s) finished.\n", t3 - t2);
    care_b200_destroy(ctx);
    return 0;
}
