// readfile.hpp -- the binary read-storage file of care-cpu
// (--save-preprocessedreads-to / --load-preprocessedreads-from;
// ChunkedReadStorage::saveToFile / loadFromFile, include/chunkedreadstorage.hpp:160-398,
// lengths as LengthStore<uint32_t>, include/lengthstorage.hpp:184-280).
//
// Layout, little-endian, in file order:
//   u64 reads; i32 longest length; i32 shortest length; u8 has qualities;
//   i32 quality bits; u64 bytes of the length, sequence, quality and
//   ambiguous sections;
//   lengths: i32 32 (bits per word), i32 bits per length, i32 shortest,
//     i32 longest, u32 mask, i64 reads, u64 words, u64 bytes, then the words:
//     length - shortest in `bits per length` bits each, packed from the most
//     significant bit of word 0 on (no words when all lengths are equal);
//   sequences: u64 pitch in 32-bit words, u64 words, then reads x pitch words
//     (2-bit codes, 16 per word, first base in the top bits);
//   qualities: u64 pitch, u64 words, then reads x pitch words (the 1/2/8-bit
//     quality encoding), or pitch 0 and no words without qualities;
//   ambiguous reads: u64 count, then the u32 read ids (the reference writes
//     them in the iteration order of its hash set; any order loads).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace careb200 {

struct ReadStorageFile {
    uint64_t n = 0;
    int min_len = 0, max_len = 0;
    bool has_quality = false;
    int quality_bits = 0;
    uint64_t seq_pitch = 0, qual_pitch = 0;      // 32-bit words per read
    std::vector<uint32_t> seq, qual;
    std::vector<int32_t> len;
    std::vector<uint32_t> ambiguous_ids;
};

// "" on success, else what is wrong with the file.
std::string read_storage_file(const std::string& path, ReadStorageFile& out);

// Writes `in` in the reference's layout (ambiguous ids in the order given).
std::string write_storage_file(const std::string& path, const ReadStorageFile& in);

}  // namespace careb200
