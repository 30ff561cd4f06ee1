// tables.hpp -- minhash tables built on the device (tables.cu).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "device.cuh"

namespace careb200 {

// Owning device array.
template <class T>
struct DevMem {
    T* p = nullptr;
    size_t n = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    DevMem(DevMem&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevMem& operator=(DevMem&& o) noexcept {
        if (this != &o) { free(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevMem() { free(); }
    cudaError_t alloc(size_t count) {
        free();
        const cudaError_t e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
        if (e == cudaSuccess) n = count; else p = nullptr;
        return e;
    }
    void free() { if (p) cudaFree(p); p = nullptr; n = 0; }
    T* release() { T* q = p; p = nullptr; n = 0; return q; }
};

// The tables of all maps: kept keys in (map, key) order with their global
// value offsets, the read ids, the open-addressing slots and descriptors.
struct DeviceTables {
    cudaError_t error = cudaErrorUnknown;
    int num_maps = 0;
    uint32_t nkeys = 0, nvalues = 0;
    size_t total_slots = 0;
    DevMem<unsigned long long> keys;
    DevMem<uint32_t> key_map, key_off, values;
    DevMem<Slot> slots;
    DevMem<TableDesc> desc;
    std::vector<uint32_t> map_first, map_keys, map_vbase, map_vcount;
};

// Tables from the resident signatures (n reads x h maps, keys of 2k bits).
// error != cudaSuccess when the device build is not possible (for example
// 2k + log2(h) > 64 bits of composite key); the caller then groups on the host.
DeviceTables build_tables_device(const unsigned long long* sig, uint32_t n, int h, int k, int threshold,
                                 cudaStream_t st);

}  // namespace careb200
