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

// The minhash-table file of care-cpu (--save-hashtables-to /
// --load-hashtables-from; OrdinaryCpuMinhasher::writeToStream / loadFromStream,
// include/ordinaryminhasher.hpp:303-339; per map CpuReadOnlyMultiValueHashTable
// and its AoSCpuSingleValueHashTable key index, include/cpuhashtable.hpp:
// 30-290, 468-685). Layout, little-endian:
//   i32 k; i32 per-map result threshold; f32 load factor; i32 maps; per map:
//   u64 values, then the u32 read ids (each key's ids a contiguous ascending
//   run); the key index: f32 load, u64 keys, u64 longest probe sequence,
//   u64 size (= keys), u64 capacity (size / load, truncated), u64 slots, then
//   the slots {u64 key, u32 first value, u32 count}: a key at
//   MurmurHash3-fmix64(key) mod capacity or the next free slot after it (keys
//   inserted in ascending order); a free slot has key all ones and value 0.
struct MinhashTablesFile {
    int k = 0, threshold = 0;
    float load = 0.8f;
    std::vector<std::vector<uint64_t>> keys;       // per map, ascending
    std::vector<std::vector<uint32_t>> offsets;    // per map, keys + 1 prefix offsets into values
    std::vector<std::vector<uint32_t>> values;     // per map, read ids
};

// Reads at most max_maps maps (the reference loads min(file, requested)).
std::string read_tables_file(const std::string& path, MinhashTablesFile& out, int max_maps);
std::string write_tables_file(const std::string& path, const MinhashTablesFile& in);

}  // namespace careb200
