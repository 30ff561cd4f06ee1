// tables.cu -- minhash tables built on the device.
//
// The content is the reference's (OrdinaryCpuMinhasher insert + groupbykey,
// include/ordinaryminhasher.hpp:376-426, include/groupbykey.hpp:99-249): per
// map, the keys that at least 2 and at most `threshold` reads share, in
// ascending key order, each with its read ids ascending. Built from the
// resident signatures of all reads:
//   1. composite keys (map << key_bits | key) with the read id as payload,
//      map-major and id-ascending, sorted by a stable LSD radix sort (8-bit
//      digits: tile histograms, one device-wide scan, stable scatter with
//      ranks from __match_any_sync within warps);
//   2. key-run heads, run lengths, the runs kept, compaction of keys,
//      per-map offsets and read ids;
//   3. per map an open-addressing index (Slot: key, offset, count; capacity
//      a power of two >= 2 keys, linear probing from murmur64(key)).
#include "tables.hpp"
#include "device.cuh"

#include <algorithm>
#include <vector>

namespace careb200 {
namespace {

constexpr int RS_THREADS = 256, RS_ITEMS = 16, RS_TILE = RS_THREADS * RS_ITEMS, RS_WARPS = RS_THREADS / 32;

__global__ void k_composite(const unsigned long long* __restrict__ sig, uint32_t n, int h, int key_bits,
                            unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals) {
    const unsigned long long N = (unsigned long long)n * h;
    for (unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j < N;
         j += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t m = (uint32_t)(j / n), i = (uint32_t)(j - (unsigned long long)m * n);
        keys[j] = ((unsigned long long)m << key_bits) | sig[(size_t)i * h + m];
        vals[j] = i;
    }
}

// digit histogram of each tile: hist[digit * ntiles + tile]
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const unsigned long long* __restrict__ keys,
                                                        unsigned long long N, int shift, uint32_t ntiles,
                                                        uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_h[256];
    const uint32_t tile = blockIdx.x;
    s_h[threadIdx.x] = 0;
    __syncthreads();
    const unsigned long long base = (unsigned long long)tile * RS_TILE;
    for (int j = threadIdx.x; j < RS_TILE; j += RS_THREADS) {
        const unsigned long long e = base + j;
        if (e < N) atomicAdd(&s_h[(keys[e] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * ntiles + tile] = s_h[threadIdx.x];
}

// exclusive scan, three kernels: per-block scan with block totals, scan of
// the totals (one block), add the scanned totals back
constexpr int SC_THREADS = 1024, SC_ITEMS = 4, SC_TILE = SC_THREADS * SC_ITEMS;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        s_warp[lane] = w;                        // inclusive prefix of warp totals
    }
    __syncthreads();
    const uint32_t before = warp ? s_warp[warp - 1] : 0u;
    *total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(SC_THREADS) k_scan_tiles(uint32_t* __restrict__ a, size_t n,
                                                           uint32_t* __restrict__ sums) {
    __shared__ uint32_t s_warp[32];
    const size_t base = (size_t)blockIdx.x * SC_TILE + (size_t)threadIdx.x * SC_ITEMS;
    uint32_t v[SC_ITEMS], t = 0;
#pragma unroll
    for (int q = 0; q < SC_ITEMS; ++q) { v[q] = base + q < n ? a[base + q] : 0u; t += v[q]; }
    uint32_t total;
    uint32_t run = block_excl_scan(t, s_warp, &total);
#pragma unroll
    for (int q = 0; q < SC_ITEMS; ++q) { if (base + q < n) a[base + q] = run; run += v[q]; }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SC_THREADS) k_scan_one(uint32_t* __restrict__ a, size_t n) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (size_t c = 0; c < n; c += SC_TILE) {
        const size_t base = c + (size_t)threadIdx.x * SC_ITEMS;
        uint32_t v[SC_ITEMS], t = 0;
#pragma unroll
        for (int q = 0; q < SC_ITEMS; ++q) { v[q] = base + q < n ? a[base + q] : 0u; t += v[q]; }
        uint32_t total;
        uint32_t run = block_excl_scan(t, s_warp, &total) + s_carry;
#pragma unroll
        for (int q = 0; q < SC_ITEMS; ++q) { if (base + q < n) a[base + q] = run; run += v[q]; }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
        __syncthreads();
    }
}

__global__ void k_scan_add(uint32_t* __restrict__ a, size_t n, const uint32_t* __restrict__ sums) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] += sums[i / SC_TILE];
}

// stable scatter of one pass: warp w holds elements [w*512, w*512+512) of
// the tile in 16 rounds of 32 consecutive elements
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const unsigned long long* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin,
                                                           unsigned long long* __restrict__ kout,
                                                           uint32_t* __restrict__ vout, unsigned long long N,
                                                           int shift, uint32_t ntiles,
                                                           const uint32_t* __restrict__ offs) {
    __shared__ uint32_t s_cnt[RS_WARPS][256];
    __shared__ uint32_t s_off[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
    for (int d = threadIdx.x; d < RS_WARPS * 256; d += RS_THREADS) (&s_cnt[0][0])[d] = 0;
    s_off[threadIdx.x] = offs[(size_t)threadIdx.x * ntiles + tile];
    __syncthreads();
    const unsigned long long base = (unsigned long long)tile * RS_TILE + (unsigned long long)warp * 32 * RS_ITEMS;
    const unsigned lt = (1u << lane) - 1u;
    unsigned long long key[RS_ITEMS];
    uint32_t val[RS_ITEMS], rank[RS_ITEMS], dig[RS_ITEMS];
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
        const unsigned long long e = base + (unsigned long long)j * 32 + lane;
        const bool ok = e < N;
        key[j] = ok ? kin[e] : 0ull;
        val[j] = ok ? vin[e] : 0u;
        dig[j] = ok ? (uint32_t)((key[j] >> shift) & 255u) : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, dig[j]);
        const uint32_t before = (dig[j] < 256u) ? s_cnt[warp][dig[j]] : 0u;
        rank[j] = before + __popc(peers & lt);
        __syncwarp();
        if (dig[j] < 256u && (peers & lt) == 0) s_cnt[warp][dig[j]] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix of the warps' counts (warp order = element order)
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
        for (int w = 0; w < RS_WARPS; ++w) { const uint32_t c = s_cnt[w][d]; s_cnt[w][d] = run; run += c; }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
        if (dig[j] < 256u) {
            const size_t pos = (size_t)s_off[dig[j]] + s_cnt[warp][dig[j]] + rank[j];
            kout[pos] = key[j];
            vout[pos] = val[j];
        }
    }
}

// run heads of the sorted composite keys
__global__ void k_heads(const unsigned long long* __restrict__ keys, unsigned long long N,
                        uint32_t* __restrict__ head) {
    for (unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j < N;
         j += (unsigned long long)gridDim.x * blockDim.x)
        head[j] = (j == 0 || keys[j] != keys[j - 1]) ? 1u : 0u;
}

// run starts (exclusive scan of heads = run index of each head)
__global__ void k_run_starts(const uint32_t* __restrict__ head_scan, const uint32_t* __restrict__ head,
                             unsigned long long N, uint32_t* __restrict__ start) {
    for (unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j < N;
         j += (unsigned long long)gridDim.x * blockDim.x)
        if (head[j]) start[head_scan[j]] = (uint32_t)j;
}

// kept runs: 2 <= length <= threshold; keep[r] in {0,1}, len[r]
__global__ void k_keep(const uint32_t* __restrict__ start, uint32_t nruns, unsigned long long N, int threshold,
                       uint32_t* __restrict__ keep, uint32_t* __restrict__ kept_len) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += gridDim.x * blockDim.x) {
        const uint32_t b = start[r];
        const uint32_t e = r + 1 < nruns ? start[r + 1] : (uint32_t)N;
        const uint32_t len = e - b;
        const bool k = len >= 2 && (int)len <= threshold;
        keep[r] = k ? 1u : 0u;
        kept_len[r] = k ? len : 0u;
    }
}

// compaction of kept runs: keys (map part dropped), value offsets, values
__global__ void k_compact(const unsigned long long* __restrict__ ckeys, const uint32_t* __restrict__ vals,
                          const uint32_t* __restrict__ start, uint32_t nruns, unsigned long long N,
                          const uint32_t* __restrict__ keep, const uint32_t* __restrict__ keep_scan,
                          const uint32_t* __restrict__ len_scan, int key_bits,
                          unsigned long long* __restrict__ out_keys, uint32_t* __restrict__ out_map,
                          uint32_t* __restrict__ out_off, uint32_t* __restrict__ out_vals) {
    const unsigned long long kmask = key_bits >= 64 ? ~0ull : ((1ull << key_bits) - 1ull);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += gridDim.x * blockDim.x) {
        if (!keep[r]) continue;
        const uint32_t b = start[r];
        const uint32_t e = r + 1 < nruns ? start[r + 1] : (uint32_t)N;
        const uint32_t s = keep_scan[r], vo = len_scan[r];
        const unsigned long long ck = ckeys[b];
        out_keys[s] = ck & kmask;
        out_map[s] = (uint32_t)(ck >> key_bits);
        out_off[s] = vo;
        for (uint32_t j = b; j < e; ++j) out_vals[vo + (j - b)] = vals[j];
    }
}

// open-addressing index: slot claimed through its count (0 = empty)
__global__ void k_slots(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ map_of,
                        const uint32_t* __restrict__ off, uint32_t nkept, uint32_t total_vals,
                        const TableDesc* __restrict__ desc, const uint32_t* __restrict__ map_first,
                        Slot* __restrict__ slots, int* __restrict__ err) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nkept; s += gridDim.x * blockDim.x) {
        const uint32_t m = map_of[s];
        const TableDesc d = desc[m];
        const uint32_t cnt = (s + 1 < nkept ? off[s + 1] : total_vals) - off[s];
        const uint32_t rel = off[s] - off[map_first[m]];          // offset within the map's values
        uint32_t pos = (uint32_t)murmur64(keys[s]) & d.mask;
        bool done = false;
        for (uint32_t probe = 0; probe <= d.mask && !done; ++probe) {
            Slot* sl = slots + d.slot_base + pos;
            if (atomicCAS(&sl->count, 0u, cnt) == 0u) {
                sl->key = keys[s];
                sl->offset = rel;
                done = true;
            }
            pos = (pos + 1) & d.mask;
        }
        if (!done) atomicOr(err, 1);
    }
}

unsigned grid_for(unsigned long long n, int threads = 256) {
    return (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>((n + threads - 1) / threads, 148ull * 32));
}

}  // namespace

// exclusive scan of a[0..n) in place; scratch >= ceil(n / SC_TILE) + 1 entries
static cudaError_t excl_scan(uint32_t* a, size_t n, uint32_t* scratch, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const size_t tiles = (n + SC_TILE - 1) / SC_TILE;
    k_scan_tiles<<<(unsigned)tiles, SC_THREADS, 0, st>>>(a, n, scratch);
    if (tiles > 1) {
        k_scan_one<<<1, SC_THREADS, 0, st>>>(scratch, tiles);
        k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, n, scratch);
    }
    return cudaGetLastError();
}

#define TCK(call)                                          \
    do {                                                   \
        const cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) { out.error = e_; return out; } \
    } while (0)

DeviceTables build_tables_device(const unsigned long long* sig, uint32_t n, int h, int k, int threshold,
                                 cudaStream_t st) {
    DeviceTables out;
    const int key_bits = 2 * k;
    int map_bits = 0;
    while ((1 << map_bits) < h) ++map_bits;
    const int sort_bits = key_bits + map_bits;
    const unsigned long long N = (unsigned long long)n * h;
    out.num_maps = h;
    if (N >= 0xFFFFFFFFull) { out.error = cudaErrorInvalidValue; return out; }
    if (sort_bits > 64) { out.error = cudaErrorInvalidValue; return out; }
    DevMem<unsigned long long> ka, kb;
    DevMem<uint32_t> va, vb;
    TCK(ka.alloc(N)); TCK(kb.alloc(N)); TCK(va.alloc(N)); TCK(vb.alloc(N));
    k_composite<<<grid_for(N), 256, 0, st>>>(sig, n, h, key_bits, ka.p, va.p);
    TCK(cudaGetLastError());
    // LSD radix sort of the composite keys (stable: ids stay ascending per key)
    const uint32_t ntiles = (uint32_t)((N + RS_TILE - 1) / RS_TILE);
    DevMem<uint32_t> hist, scr;
    const size_t hn = (size_t)256 * ntiles;
    TCK(hist.alloc(hn));
    TCK(scr.alloc(std::max<size_t>((hn + SC_TILE - 1) / SC_TILE, (N + SC_TILE - 1) / SC_TILE) + 2));
    for (int shift = 0; shift < sort_bits; shift += 8) {
        k_rs_hist<<<ntiles, RS_THREADS, 0, st>>>(ka.p, N, shift, ntiles, hist.p);
        TCK(cudaGetLastError());
        TCK(excl_scan(hist.p, hn, scr.p, st));
        k_rs_scatter<<<ntiles, RS_THREADS, 0, st>>>(ka.p, va.p, kb.p, vb.p, N, shift, ntiles, hist.p);
        TCK(cudaGetLastError());
        std::swap(ka.p, kb.p);
        std::swap(va.p, vb.p);
    }
    // runs of equal composite keys, the kept ones, compaction
    DevMem<uint32_t> head, hscan, start;
    TCK(head.alloc(N)); TCK(hscan.alloc(N));
    k_heads<<<grid_for(N), 256, 0, st>>>(ka.p, N, head.p);
    TCK(cudaGetLastError());
    TCK(cudaMemcpyAsync(hscan.p, head.p, N * 4, cudaMemcpyDeviceToDevice, st));
    TCK(excl_scan(hscan.p, N, scr.p, st));
    uint32_t last_scan = 0, last_head = 0;
    TCK(cudaMemcpyAsync(&last_scan, hscan.p + N - 1, 4, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(&last_head, head.p + N - 1, 4, cudaMemcpyDeviceToHost, st));
    TCK(cudaStreamSynchronize(st));
    const uint32_t nruns = last_scan + last_head;
    TCK(start.alloc(nruns));
    k_run_starts<<<grid_for(N), 256, 0, st>>>(hscan.p, head.p, N, start.p);
    TCK(cudaGetLastError());
    head.free(); hscan.free();
    DevMem<uint32_t> keep, kscan, klen;
    TCK(keep.alloc(nruns)); TCK(kscan.alloc(nruns)); TCK(klen.alloc(nruns));
    k_keep<<<grid_for(nruns), 256, 0, st>>>(start.p, nruns, N, threshold, keep.p, klen.p);
    TCK(cudaGetLastError());
    TCK(cudaMemcpyAsync(kscan.p, keep.p, (size_t)nruns * 4, cudaMemcpyDeviceToDevice, st));
    uint32_t lastk = 0, lastlen = 0;
    TCK(cudaMemcpyAsync(&lastk, keep.p + nruns - 1, 4, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(&lastlen, klen.p + nruns - 1, 4, cudaMemcpyDeviceToHost, st));
    TCK(excl_scan(kscan.p, nruns, scr.p, st));
    TCK(excl_scan(klen.p, nruns, scr.p, st));
    uint32_t kscan_last = 0, klen_last = 0;
    TCK(cudaMemcpyAsync(&kscan_last, kscan.p + nruns - 1, 4, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(&klen_last, klen.p + nruns - 1, 4, cudaMemcpyDeviceToHost, st));
    TCK(cudaStreamSynchronize(st));
    const uint32_t nkept = kscan_last + lastk, nvals = klen_last + lastlen;
    TCK(out.keys.alloc(std::max<uint32_t>(nkept, 1)));
    TCK(out.key_map.alloc(std::max<uint32_t>(nkept, 1)));
    TCK(out.key_off.alloc(std::max<uint32_t>(nkept, 1)));
    TCK(out.values.alloc(std::max<uint32_t>(nvals, 1)));
    k_compact<<<grid_for(nruns), 256, 0, st>>>(ka.p, va.p, start.p, nruns, N, keep.p, kscan.p, klen.p, key_bits,
                                               out.keys.p, out.key_map.p, out.key_off.p, out.values.p);
    TCK(cudaGetLastError());
    ka.free(); kb.free(); va.free(); vb.free(); start.free(); keep.free(); kscan.free(); klen.free();
    // per map: first kept key, key count, value count (from the compacted map ids)
    std::vector<uint32_t> kmap(nkept), koff(nkept);
    if (nkept) {
        TCK(cudaMemcpyAsync(kmap.data(), out.key_map.p, (size_t)nkept * 4, cudaMemcpyDeviceToHost, st));
        TCK(cudaMemcpyAsync(koff.data(), out.key_off.p, (size_t)nkept * 4, cudaMemcpyDeviceToHost, st));
        TCK(cudaStreamSynchronize(st));
    }
    out.map_first.assign(h, 0);
    out.map_keys.assign(h, 0);
    {
        size_t s = 0;
        for (int m = 0; m < h; ++m) {
            out.map_first[m] = (uint32_t)s;
            while (s < nkept && kmap[s] == (uint32_t)m) ++s;
            out.map_keys[m] = (uint32_t)s - out.map_first[m];
        }
    }
    out.map_vbase.assign(h, 0);
    out.map_vcount.assign(h, 0);
    for (int m = 0; m < h; ++m) {
        const uint32_t f = out.map_first[m], c = out.map_keys[m];
        out.map_vbase[m] = c ? koff[f] : (f < nkept ? koff[f] : nvals);
        const uint32_t e = f + c < nkept ? koff[f + c] : nvals;
        out.map_vcount[m] = c ? e - out.map_vbase[m] : 0;
    }
    // slots
    std::vector<TableDesc> desc(h);
    size_t total_slots = 0;
    for (int m = 0; m < h; ++m) {
        size_t cap = 16;
        while (cap < 2 * (size_t)out.map_keys[m]) cap <<= 1;
        desc[m].slot_base = total_slots;
        desc[m].value_base = out.map_vbase[m];
        desc[m].mask = (uint32_t)(cap - 1);
        desc[m].pad = 0;
        total_slots += cap;
    }
    TCK(out.slots.alloc(total_slots));
    TCK(out.desc.alloc(h));
    TCK(cudaMemsetAsync(out.slots.p, 0, total_slots * sizeof(Slot), st));
    TCK(cudaMemcpyAsync(out.desc.p, desc.data(), h * sizeof(TableDesc), cudaMemcpyHostToDevice, st));
    DevMem<uint32_t> mfirst;
    DevMem<int> err;
    TCK(mfirst.alloc(h)); TCK(err.alloc(1));
    TCK(cudaMemcpyAsync(mfirst.p, out.map_first.data(), h * 4, cudaMemcpyHostToDevice, st));
    TCK(cudaMemsetAsync(err.p, 0, 4, st));
    if (nkept) {
        k_slots<<<grid_for(nkept), 256, 0, st>>>(out.keys.p, out.key_map.p, out.key_off.p, nkept, nvals, out.desc.p,
                                                 mfirst.p, out.slots.p, err.p);
        TCK(cudaGetLastError());
    }
    int herr = 0;
    TCK(cudaMemcpyAsync(&herr, err.p, 4, cudaMemcpyDeviceToHost, st));
    TCK(cudaStreamSynchronize(st));
    if (herr) { out.error = cudaErrorUnknown; return out; }
    out.nkeys = nkept;
    out.nvalues = nvals;
    out.total_slots = total_slots;
    out.error = cudaSuccess;
    return out;
}

}  // namespace careb200
