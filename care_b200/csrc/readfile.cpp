// readfile.cpp -- care-cpu's binary read-storage file (layout in readfile.hpp).
#include "readfile.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>

namespace careb200 {
namespace {

// Bits per stored length for lengths in [lo, hi]: 0 when all are equal, else
// the exponent of the power of two above hi - lo (LengthStore's constructor,
// include/lengthstorage.hpp:20-44).
int length_bits(int lo, int hi) {
    uint32_t v = (uint32_t)(hi - lo);
    if (v == 0) return 0;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    v += 1;                                   // a power of two
    int b = 0;
    while ((1ull << b) < v) ++b;
    return b;
}

uint64_t length_words(int bits, uint64_t n) { return (bits * n + 31) / 32; }

template <class T>
bool get(std::istream& s, T& v) { return (bool)s.read(reinterpret_cast<char*>(&v), sizeof(T)); }
template <class T>
void put(std::ostream& s, const T& v) { s.write(reinterpret_cast<const char*>(&v), sizeof(T)); }

// Bytes left in the stream: sizes read from a file are checked against it
// before anything is allocated.
uint64_t remaining(std::istream& s) {
    const auto here = s.tellg();
    s.seekg(0, std::ios::end);
    const auto end = s.tellg();
    s.seekg(here);
    return (here < 0 || end < here) ? 0 : (uint64_t)(end - here);
}

bool get_words(std::istream& s, std::vector<uint32_t>& v, uint64_t count) {
    if (count > remaining(s) / 4) return false;
    v.resize(count);
    return count == 0 || (bool)s.read(reinterpret_cast<char*>(v.data()), count * 4);
}

// MurmurHash3's 64-bit finalizer (fmix64), the key hash of the index.
uint64_t fmix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

#pragma pack(push, 1)
struct IndexSlot {
    uint64_t key;
    uint32_t first, count;
};
#pragma pack(pop)
static_assert(sizeof(IndexSlot) == 16, "index slot layout");

}  // namespace

std::string read_storage_file(const std::string& path, ReadStorageFile& f) {
    std::ifstream s(path, std::ios::binary);
    if (!s) return "cannot open " + path;
    const std::string trunc = path + ": truncated or not a read-storage file";
    uint64_t n = 0, bytes[4];
    int hi = 0, lo = 0, qbits = 0;
    uint8_t hasq = 0;
    if (!get(s, n) || !get(s, hi) || !get(s, lo) || !get(s, hasq) || !get(s, qbits)) return trunc;
    for (auto& b : bytes) if (!get(s, b)) return trunc;
    if (n == 0 || n > std::numeric_limits<uint32_t>::max() || n > remaining(s)) return path + ": read count out of range";

    // lengths
    int word_bits = 0, bits = 0, mn = 0, mx = 0;
    uint32_t mask = 0;
    int64_t elems = 0;
    uint64_t raw_words = 0, raw_bytes = 0;
    if (!get(s, word_bits) || !get(s, bits) || !get(s, mn) || !get(s, mx) || !get(s, mask) || !get(s, elems) ||
        !get(s, raw_words) || !get(s, raw_bytes))
        return trunc;
    if (word_bits != 32 || elems != (int64_t)n || raw_bytes != raw_words * 4 || mn < 1 || mx < mn ||
        bits != length_bits(mn, mx) || raw_words < length_words(bits, n))
        return path + ": inconsistent length section";
    std::vector<uint32_t> lw;
    if (!get_words(s, lw, raw_words)) return trunc;
    f.len.assign(n, mn);
    if (bits > 0) {
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t v = 0;
            for (int j = 0; j < bits; ++j) {
                const uint64_t g = (uint64_t)bits * i + j;           // bit g counted from the top of word 0
                v = (v << 1) | ((lw[g >> 5] >> (31 - (g & 31))) & 1u);
            }
            f.len[i] = mn + (int)v;
            if (f.len[i] > mx) return path + ": stored length above the longest";
        }
    }

    // sequences
    uint64_t sp = 0, sn = 0;
    if (!get(s, sp) || !get(s, sn)) return trunc;
    if (sp == 0 || sp > (1u << 20) || sn != n * sp || (uint64_t)mx > 16 * sp) return path + ": inconsistent sequence section";
    if (!get_words(s, f.seq, sn)) return trunc;

    // qualities
    uint64_t qp = 0, qn = 0;
    if (!get(s, qp) || !get(s, qn)) return trunc;
    if (hasq) {
        if (qbits != 1 && qbits != 2 && qbits != 8) return path + ": quality bits must be 1, 2 or 8";
        const uint64_t per = 32 / qbits;
        if (qp > (1u << 20) || qn != n * qp || (uint64_t)mx > per * qp) return path + ": inconsistent quality section";
        if (!get_words(s, f.qual, qn)) return trunc;
    } else {
        if (qn != 0) s.seekg((std::streamoff)(qn * 4), std::ios::cur);
        f.qual.clear();
        qp = 0;
    }

    // ambiguous reads
    uint64_t na = 0;
    if (!get(s, na) || na > n) return trunc;
    if (!get_words(s, f.ambiguous_ids, na)) return trunc;
    for (uint32_t id : f.ambiguous_ids)
        if (id >= n) return path + ": ambiguous read id out of range";

    f.n = n;
    f.min_len = mn;
    f.max_len = mx;
    f.has_quality = hasq != 0;
    f.quality_bits = qbits;
    f.seq_pitch = sp;
    f.qual_pitch = qp;
    return "";
}

std::string write_storage_file(const std::string& path, const ReadStorageFile& f) {
    if (f.n == 0 || f.len.size() != f.n || f.seq.size() != f.n * f.seq_pitch ||
        (f.has_quality && f.qual.size() != f.n * f.qual_pitch))
        return "inconsistent read storage";
    std::ofstream s(path, std::ios::binary | std::ios::trunc);
    if (!s) return "cannot create " + path;
    const int bits = length_bits(f.min_len, f.max_len);
    std::vector<uint32_t> lw(bits ? length_words(bits, f.n) : 0, 0u);
    for (uint64_t i = 0; bits && i < f.n; ++i) {
        const uint32_t v = (uint32_t)(f.len[i] - f.min_len);
        for (int j = 0; j < bits; ++j) {
            const uint64_t g = (uint64_t)bits * i + j;
            if ((v >> (bits - 1 - j)) & 1u) lw[g >> 5] |= 1u << (31 - (g & 31));
        }
    }
    const uint64_t qp = f.has_quality ? f.qual_pitch : 0, qn = f.has_quality ? f.qual.size() : 0;
    const uint64_t na = f.ambiguous_ids.size();
    const uint64_t len_bytes = 4 * 4 + 4 + 8 + 8 + 8 + lw.size() * 4;
    const uint64_t seq_bytes = 16 + f.seq.size() * 4;
    const uint64_t qual_bytes = 16 + qn * 4;
    const uint64_t amb_bytes = 8 + na * 4;

    put(s, f.n);
    put(s, f.max_len);                       // the reference writes the longest length first
    put(s, f.min_len);
    put(s, (uint8_t)(f.has_quality ? 1 : 0));
    put(s, f.quality_bits);
    put(s, len_bytes); put(s, seq_bytes); put(s, qual_bytes); put(s, amb_bytes);

    put(s, (int)32);
    put(s, bits);
    put(s, f.min_len);
    put(s, f.max_len);
    put(s, (uint32_t)(bits ? (1u << bits) - 1u : 0u));
    put(s, (int64_t)f.n);
    put(s, (uint64_t)lw.size());
    put(s, (uint64_t)lw.size() * 4);
    if (!lw.empty()) s.write(reinterpret_cast<const char*>(lw.data()), lw.size() * 4);

    put(s, f.seq_pitch);
    put(s, (uint64_t)f.seq.size());
    s.write(reinterpret_cast<const char*>(f.seq.data()), f.seq.size() * 4);

    put(s, qp);
    put(s, qn);
    if (qn) s.write(reinterpret_cast<const char*>(f.qual.data()), qn * 4);

    put(s, na);
    if (na) s.write(reinterpret_cast<const char*>(f.ambiguous_ids.data()), na * 4);
    if (!s) return "write failed: " + path;
    return "";
}

std::string read_tables_file(const std::string& path, MinhashTablesFile& t, int max_maps) {
    std::ifstream s(path, std::ios::binary);
    if (!s) return "cannot open " + path;
    const std::string trunc = path + ": truncated or not a minhash-table file";
    int k = 0, thr = 0, maps = 0;
    float lf = 0.f;
    if (!get(s, k) || !get(s, thr) || !get(s, lf) || !get(s, maps)) return trunc;
    if (k < 1 || k > 32 || maps < 1) return path + ": bad header";
    const int use = std::min(maps, max_maps);
    t = MinhashTablesFile{};
    t.k = k;
    t.threshold = thr;
    t.load = lf;
    for (int m = 0; m < use; ++m) {
        uint64_t nv = 0;
        std::vector<uint32_t> vals;
        if (!get(s, nv) || !get_words(s, vals, nv)) return trunc;
        float load = 0.f;
        uint64_t nk = 0, probes = 0, size = 0, cap = 0, nslots = 0;
        if (!get(s, load) || !get(s, nk) || !get(s, probes) || !get(s, size) || !get(s, cap) || !get(s, nslots))
            return trunc;
        if (nslots != cap || nk > cap || nslots > remaining(s) / sizeof(IndexSlot)) return path + ": inconsistent key index";
        std::vector<IndexSlot> slots(nslots);
        if (nslots && !s.read(reinterpret_cast<char*>(slots.data()), nslots * sizeof(IndexSlot))) return trunc;
        std::vector<IndexSlot> used;
        for (const IndexSlot& e : slots) {
            if (e.key == ~0ull) continue;
            if ((uint64_t)e.first + e.count > nv) return path + ": key index points past the values";
            used.push_back(e);
        }
        if (used.size() != nk) return path + ": key count differs from the index";
        std::sort(used.begin(), used.end(), [](const IndexSlot& a, const IndexSlot& b) { return a.key < b.key; });
        std::vector<uint64_t> keys;
        std::vector<uint32_t> off{0}, v;
        for (const IndexSlot& e : used) {
            keys.push_back(e.key);
            v.insert(v.end(), vals.begin() + e.first, vals.begin() + e.first + e.count);
            off.push_back((uint32_t)v.size());
        }
        t.keys.push_back(std::move(keys));
        t.offsets.push_back(std::move(off));
        t.values.push_back(std::move(v));
    }
    return "";
}

std::string write_tables_file(const std::string& path, const MinhashTablesFile& t) {
    const int maps = (int)t.keys.size();
    if (maps < 1 || t.offsets.size() != t.keys.size() || t.values.size() != t.keys.size())
        return "inconsistent tables";
    std::ofstream s(path, std::ios::binary | std::ios::trunc);
    if (!s) return "cannot create " + path;
    put(s, t.k);
    put(s, t.threshold);
    put(s, t.load);
    put(s, maps);
    for (int m = 0; m < maps; ++m) {
        const auto& keys = t.keys[m];
        const auto& off = t.offsets[m];
        const uint64_t nv = keys.empty() ? 0 : off[keys.size()];
        put(s, nv);
        if (nv) s.write(reinterpret_cast<const char*>(t.values[m].data()), nv * 4);
        // the key index as the reference builds it: size = keys, capacity
        // size / load in float, keys inserted in ascending order with linear probing
        const uint64_t size = keys.size();
        const uint64_t cap = (uint64_t)((float)size / t.load);
        if (size > cap) return "load factor above 1";
        // a free slot: key all ones, value {0, 0} (the reference's
        // numeric_limits max of a pair value is a value-initialised pair)
        std::vector<IndexSlot> slots(cap, IndexSlot{~0ull, 0u, 0u});
        uint64_t probes_max = 0;
        for (size_t i = 0; i < keys.size(); ++i) {
            uint64_t pos = fmix64(keys[i]) % cap, probes = 0;
            while (slots[pos].key != ~0ull) {
                if (++pos == cap) pos = 0;
                ++probes;
            }
            slots[pos] = IndexSlot{keys[i], off[i], off[i + 1] - off[i]};
            probes_max = std::max(probes_max, probes);
        }
        put(s, t.load);
        put(s, size);
        put(s, probes_max);
        put(s, size);
        put(s, cap);
        put(s, cap);
        if (cap) s.write(reinterpret_cast<const char*>(slots.data()), cap * sizeof(IndexSlot));
    }
    if (!s) return "write failed: " + path;
    return "";
}

}  // namespace careb200
