// hostio.hpp -- host side of the correction path: input parsing and read
// preprocessing (STEP1 of care-cpu) and output construction (STEP3).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace careb200 {

// Parsed reads with the reference's preprocessing applied
// (chunkedreadstorageconstruction.hpp:29-485).
struct HostReads {
    uint32_t n = 0;
    int min_len = 0, max_len = 0;
    int seq_pitch = 0, qual_pitch = 0, quality_bits = 8;
    bool has_quality = false;
    bool fasta = false;
    std::vector<uint32_t> seq;        // n * seq_pitch
    std::vector<uint32_t> qual;       // n * qual_pitch
    std::vector<int32_t> len;
    std::vector<uint8_t> ambig;
    std::vector<uint32_t> ambiguous_ids;
    // original records for output: header, sequence, quality, NUL separated
    std::vector<char> text;
    std::vector<size_t> rec_off;
    // or (records parsed on the device) offsets into the input files' bytes:
    // header (after '@' / '>', without the line end), sequence, quality
    // (both of the read's length)
    const char* raw = nullptr;
    std::vector<uint64_t> rec_h, rec_s, rec_q;
    std::vector<uint32_t> rec_hl;
};

// Returns an empty string on success, else an error message.
std::string load_reads(const std::vector<std::string>& files, bool paired_end, bool use_quality,
                       int quality_bits, HostReads& out);
// The same with at most `threads` threads (1: a single sequential scan).
std::string load_reads_threads(const std::vector<std::string>& files, bool paired_end, bool use_quality,
                               int quality_bits, HostReads& out, unsigned threads);

void encode_2bit(const char* s, int len, uint32_t* out);
void encode_quality(const char* q, int len, int bits, uint32_t* out);
int quality_ints(int len, int bits);

// Quality weight table of the reference's QualityScoreConversion
// (qualityscoreweights.hpp:16-31).
void quality_weights(float* w256);

// One correction outcome in host memory.
struct HostCorrections {
    uint32_t first = 0, count = 0;
    int max_len = 0;
    const uint8_t* status = nullptr;
    const int32_t* nedits = nullptr;
    const char* seq = nullptr;
    uint64_t ncand = 0;
    const uint32_t* cand_id = nullptr;
    const uint8_t* cand_use_edits = nullptr;
    const char* cand_seq = nullptr;
};

// Merge corrections with the original reads and write the output file
// (correctionresultoutput.cpp:30-440, combiner :730-1020; writer
// readlibraryio.cpp:61-80). Returns an empty string on success.
std::string write_corrected(const HostReads& reads, const HostCorrections& c, bool quality_labels,
                            const std::string& path);

}  // namespace careb200
