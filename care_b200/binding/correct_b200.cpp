// correct_b200.cpp -- CARE's STEP2 served by care-b200, inside the reference's
// own care-cpu program.
//
// This file is the binding a CARE maintainer adds: a definition of
// care::cpu::correct_cpu (declared in include/correct_cpu.hpp of the
// reference, implemented by src/correct_cpu.cpp:47-348) with the same
// arguments and the same result -- the serialized EncodedTempCorrectedSequence
// records (include/correctedsequence.hpp:148-340) that STEP3 sorts, merges and
// writes. Compiled with -Dcorrect_cpu=correct_b200, both this file and the
// reference's src/dispatch_care_correct_cpu.cpp see the name correct_b200, so
// the dispatch's call (src/dispatch_care_correct_cpu.cpp:159-163) lands here
// while its STEP1 (read storage, minhasher) and STEP3 stay the reference's.
// oracle/Makefile (target ref-b200) builds that program from the reference's
// sources and this file, linked to libcareb200.so.
#include <correct_cpu.hpp>
#include <cpuminhasher.hpp>
#include <cpureadstorage.hpp>
#include <options.hpp>
#include <qualityscorecompression.hpp>
#include <sequencehelpers.hpp>
#include <serializedobjectstorage.hpp>

#include <care_b200.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace care {
namespace cpu {

namespace {

struct Ctx {
    care_b200_ctx* p = nullptr;
    ~Ctx() { if (p) care_b200_destroy(p); }
    void check(int rc, const char* what) const {
        if (rc != CARE_B200_OK)
            throw std::runtime_error(std::string("care-b200 ") + what + " failed (" + std::to_string(rc) +
                                     "): " + (p ? care_b200_last_error(p) : ""));
    }
};

}  // namespace

SerializedObjectStorage correct_cpu(const ProgramOptions& po, CpuMinhasher& minhasher, CpuReadStorage& readStorage) {
    if (po.correctionType != CorrectionType::Classic)
        throw std::runtime_error("care-b200 serves the classic correction (--correctionType 0)");

    care_b200_options o;
    care_b200_default_options(&o);
    o.kmerlength = minhasher.getKmerSize();
    o.num_maps = minhasher.getNumberOfMaps();
    o.min_overlap = po.min_overlap;
    o.max_error_rate = po.maxErrorRate;
    o.min_overlap_ratio = po.min_overlap_ratio;
    o.estimated_errorrate = po.estimatedErrorrate;
    o.estimated_coverage = po.estimatedCoverage;
    o.m_coverage = po.m_coverage;
    o.paired_filter_threshold = po.pairedFilterThreshold;
    o.new_columns_to_correct = po.new_columns_to_correct;
    o.use_quality = po.useQualityScores && readStorage.canUseQualityScores();
    o.quality_bits = o.use_quality ? readStorage.getQualityBits() : po.qualityScoreBits;
    o.exclude_ambiguous = po.excludeAmbiguousReads;
    o.correct_candidates = po.correctCandidates;
    o.paired_end = po.pairType == SequencePairType::PairedEnd;
    o.threads = po.threads;

    Ctx ctx;
    ctx.check(care_b200_create(&o, &ctx.p), "create");

    // read-storage handle: the reads, lengths, encoded qualities and ambiguous
    // ids of the reference's CpuReadStorage, copied once to the device
    const read_number n = readStorage.getNumberOfReads();
    const int maxLen = readStorage.getSequenceLengthUpperBound();
    const std::size_t pitch = SequenceHelpers::getEncodedNumInts2Bit(maxLen);
    const std::size_t qpitch = o.use_quality ? QualityCompressionHelper::getNumInts(maxLen, o.quality_bits) : 0;
    std::vector<unsigned int> seq((std::size_t)n * pitch), qual((std::size_t)n * qpitch);
    std::vector<int> len(n);
    std::vector<read_number> ids;
    constexpr read_number chunk = read_number(1) << 24;
    for (read_number b = 0; b < n; b += chunk) {
        const int m = (int)std::min<read_number>(chunk, n - b);
        readStorage.gatherContiguousSequences(seq.data() + (std::size_t)b * pitch, pitch, b, m);
        if (o.use_quality)
            readStorage.gatherContiguousEncodedQualities(qual.data() + (std::size_t)b * qpitch, qpitch, b, m);
        ids.resize(m);
        std::iota(ids.begin(), ids.end(), b);
        readStorage.gatherSequenceLengths(len.data() + b, ids.data(), m);
    }
    std::vector<read_number> ambiguous(readStorage.getNumberOfReadsWithN());
    if (!ambiguous.empty()) readStorage.getIdsOfAmbiguousReads(ambiguous.data());
    ctx.check(care_b200_upload_reads(ctx.p, seq.data(), pitch, len.data(), o.use_quality ? qual.data() : nullptr,
                                     qpitch, ambiguous.data(), ambiguous.size(), n),
              "upload_reads");
    std::vector<unsigned int>().swap(seq);
    std::vector<unsigned int>().swap(qual);

    // minhasher handle: tables with the reference's contents built on the
    // device; tables whose per-map threshold is not the one the coverage gives
    // (loaded from a file) are handed over through the reference's own table
    // file instead
    if (care_b200_result_threshold(ctx.p) == minhasher.getNumResultsPerMapThreshold() ||
        !minhasher.canWriteToStream()) {
        ctx.check(care_b200_build_tables(ctx.p), "build_tables");
    } else {
        const std::string path = po.tempdirectory + "/care_b200_tables.tmp";
        {
            std::ofstream os(path, std::ios::binary);
            minhasher.writeToStream(os);
            if (!os) throw std::runtime_error("cannot write " + path);
        }
        const int rc = care_b200_load_hashtables(ctx.p, path.c_str());
        std::remove(path.c_str());
        ctx.check(rc, "load_hashtables");
    }

    care_b200_results res;
    ctx.check(care_b200_correct_range(ctx.p, 0, n, &res), "correct_range");
    std::size_t need = 0;
    ctx.check(care_b200_serialize_results(ctx.p, &res, nullptr, 0, &need), "serialize_results");
    std::vector<std::uint8_t> blob(need);
    ctx.check(care_b200_serialize_results(ctx.p, &res, blob.data(), blob.size(), &need), "serialize_results");

    // the partial-results budget of the reference (src/correct_cpu.cpp:52-95):
    // host memory left by the read storage and minhasher, minus 2 GB, split
    // 3:1 between record bytes and offsets
    std::size_t avail = po.memoryTotalLimit;
    const std::size_t used = readStorage.getMemoryInfo().host + minhasher.getMemoryInfo().host;
    avail = avail > used ? avail - used : 0;
    const std::size_t forResults = avail > (std::size_t(2) << 30) ? avail - (std::size_t(2) << 30) : 0;
    SerializedObjectStorage partialResults(forResults * 0.75, forResults * 0.25, po.tempdirectory + "/");

    // one record: read id (4 bytes), flags (4 bytes; low 29 bits = payload
    // bytes), payload
    for (std::size_t p = 0; p < need;) {
        std::uint32_t flags;
        std::memcpy(&flags, blob.data() + p + 4, 4);
        const std::size_t size = 8 + (flags & ((1u << 29) - 1));
        partialResults.insert(blob.data() + p, blob.data() + p + size);
        p += size;
    }
    return partialResults;
}

}  // namespace cpu
}  // namespace care
