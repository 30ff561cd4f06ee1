// parse.hpp -- STEP1 read parsing and encoding on the device.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace careb200 {

// Reads parsed and encoded on the device. The device arrays are allocated
// with cudaMalloc and owned by the caller afterwards.
struct DeviceParsed {
    uint32_t n = 0;
    int min_len = 0, max_len = 0, seq_pitch = 0, qual_pitch = 0;
    bool fasta = false, has_quality = false;
    uint32_t* seq = nullptr;          // n * seq_pitch, 2-bit MSB-first (zero padded)
    uint32_t* qual = nullptr;         // n * qual_pitch (has_quality)
    int32_t* len = nullptr;
    uint8_t* ambig = nullptr;
    // host copies for the output writer and the serializer
    std::vector<uint32_t> h_seq;
    std::vector<int32_t> h_len;
    std::vector<uint8_t> h_ambig;
    std::vector<uint64_t> rec_h, rec_s, rec_q;   // header (after '@' / '>'), sequence, quality offsets
    std::vector<uint32_t> rec_hl;
    void release();
};

// Parses the files' bytes (concatenated in `text`, file f starting at
// file_begin[f], each file ending with '\n'; `text` pinned host memory of
// text_bytes) as the host parse (hostio.cpp load_reads_threads) does for
// strict 4-line FASTQ or 2-line FASTA records, with the reference's
// preprocessing (chunkedreadstorageconstruction.hpp:67-92: lower case upper-
// cased, other characters A, C, G, T in turn, the turn counter restarting at
// every 65,536-read parser batch) and quality encoding
// (qualityscorecompression.hpp:90-119). Returns "" on success, "irregular"
// when the records are not in that strict layout (the host parse reads
// those), or an error message.
std::string parse_on_device(const char* text, size_t text_bytes, const size_t* file_begin, int num_files,
                            bool paired_end, bool use_quality, int quality_bits, int max_len_limit,
                            cudaStream_t st, DeviceParsed& out);

}  // namespace careb200
