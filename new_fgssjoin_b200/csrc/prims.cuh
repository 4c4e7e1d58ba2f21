// prims.cuh -- device-wide exclusive scan and stable LSD radix sort.
//
// The reference calls thrust::exclusive_scan in 1e9-element chunks plus a
// carry kernel (include/fgssjoin/scan.cuh:13-105).  Here the scan is a
// three-phase reduce-then-scan of our own (tile scan, one-CTA scan of tile
// totals, carry add) and the sort an 8-bit-digit LSD radix sort with
// warp-match stable ranking.  Both can take their element count from device
// memory (`d_n`), so a captured CUDA graph can run them on data-dependent
// sizes; `n_cap` sizes the grid.
#pragma once

#include "common.cuh"
#include "ctx.h"

namespace fgss {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

// `in` may alias `out` (in-place scans): each element is read and written by
// the same thread, the read before the block's barrier and the write after.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const T* in, T* out, T* tile_sums,
                                                              uint64_t n_cap, const uint64_t* d_n) {
    __shared__ T wsum[33];
    const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        uint64_t idx = base + i;
        v[i] = idx < n ? in[idx] : T(0);
        s += v[i];
    }
    T total;
    T pre = block_excl_scan<T>(s, wsum, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        uint64_t idx = base + i;
        T x = v[i];
        if (idx < n) out[idx] = pre;
        pre += x;
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One CTA scans the tile totals in place (exclusive) and writes the grand total.
template <typename T>
__global__ void __launch_bounds__(1024) k_scan_totals(T* sums, uint64_t ntiles_cap, uint64_t n_cap,
                                                      const uint64_t* d_n, T* grand_total) {
    __shared__ T wsum[33];
    const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
    const uint64_t ntiles = n == 0 ? 0 : (n + kScanTile - 1) / kScanTile;
    T carry = 0;
    for (uint64_t b = 0; b < ntiles; b += blockDim.x) {
        uint64_t i = b + threadIdx.x;
        T x = i < ntiles ? sums[i] : T(0);
        T tot;
        T pre = block_excl_scan<T>(x, wsum, &tot);
        if (i < ntiles) sums[i] = pre + carry;
        carry += tot;
    }
    if (threadIdx.x == 0 && grand_total) *grand_total = carry;
    (void)ntiles_cap;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_add(T* out, const T* __restrict__ sums, uint64_t n_cap,
                                                           const uint64_t* d_n) {
    const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
    const T c = sums[blockIdx.x];
    if (c == 0) return;
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {
        uint64_t idx = base + i;
        if (idx < n) out[idx] += c;
    }
}

// Exclusive scan of n_cap (or *d_n) elements; optional grand total to `total` (device).
template <typename T>
void exclusive_scan(Ctx& c, const T* in, T* out, uint64_t n_cap, const uint64_t* d_n, T* total,
                    const char* tag = "scan") {
    uint64_t ntiles = n_cap == 0 ? 1 : (n_cap + kScanTile - 1) / kScanTile;
    T* sums = c.devT<T>(std::string(tag) + ".tiles", ntiles + 1);
    k_scan_tiles<T><<<(unsigned)ntiles, kScanThreads, 0, c.stream>>>(in, out, sums, n_cap, d_n);
    FGSS_LAUNCH_CK();
    k_scan_totals<T><<<1, 1024, 0, c.stream>>>(sums, ntiles, n_cap, d_n, total);
    FGSS_LAUNCH_CK();
    k_scan_add<T><<<(unsigned)ntiles, kScanThreads, 0, c.stream>>>(out, sums, n_cap, d_n);
    FGSS_LAUNCH_CK();
}

// ------------------------------------------------------------- radix sort

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kSortWarps = kSortThreads / 32;

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
    return (uint32_t)((k >> shift) & 0xffu);
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const K* __restrict__ keys, uint32_t* hist,
                                                            uint64_t n_cap, const uint64_t* d_n, int shift,
                                                            uint32_t ntiles_cap) {
    __shared__ uint32_t h[kSortWarps][256];
    const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
    const uint32_t wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortRounds; r++) {
        uint64_t idx = base + (uint64_t)r * kSortThreads + threadIdx.x;
        if (idx < n) atomicAdd(&h[wid][digit_of(keys[idx], shift)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) s += h[w][d];
        hist[(uint64_t)d * ntiles_cap + blockIdx.x] = s;
    }
}

template <typename K, typename V>
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const K* __restrict__ kin, K* kout,
                                                               const V* __restrict__ vin, V* vout,
                                                               const uint32_t* __restrict__ offs, uint64_t n_cap,
                                                               const uint64_t* d_n, int shift, uint32_t ntiles_cap) {
    __shared__ uint32_t run[256];               // items of each digit placed so far in this tile
    __shared__ uint32_t wcnt[kSortWarps][256];  // per-round, per-warp digit counts -> prefixes
    __shared__ uint32_t gbase[256];
    const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        run[d] = 0;
        gbase[d] = offs[(uint64_t)d * ntiles_cap + blockIdx.x];
    }
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    const uint32_t lt = lanemask_lt();
    for (int r = 0; r < kSortRounds; r++) {
        uint64_t idx = base + (uint64_t)r * kSortThreads + threadIdx.x;
        bool valid = idx < n;
        K k = valid ? kin[idx] : K(0);
        V v = V();
        if (valid && vin) v = vin[idx];
        uint32_t d = valid ? digit_of(k, shift) : 256u;
        uint32_t peers = __match_any_sync(kFull, d);
        uint32_t lrank = __popc(peers & lt);
        uint32_t leader = __ffs(peers) - 1;
        if (valid && lane == leader) wcnt[wid][d] = __popc(peers);
        __syncthreads();
        for (int dd = threadIdx.x; dd < 256; dd += kSortThreads) {
            uint32_t acc = run[dd];
#pragma unroll
            for (int w = 0; w < kSortWarps; w++) {
                uint32_t cc = wcnt[w][dd];
                wcnt[w][dd] = acc;
                acc += cc;
            }
            run[dd] = acc;
        }
        __syncthreads();
        if (valid) {
            uint32_t dst = gbase[d] + wcnt[wid][d] + lrank;
            kout[dst] = k;
            if (vin) vout[dst] = v;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&wcnt[0][0])[i] = 0;
        __syncthreads();
    }
}

// Stable sort of (keys, values) by key bits [begin_bit, end_bit).  Ping-pongs
// between the given arrays and pool scratch; the sorted data ends in the
// given arrays.  `values` may be null.  Element count below 2^32.
template <typename K, typename V>
void radix_sort(Ctx& c, K* keys, V* values, uint64_t n_cap, const uint64_t* d_n, int begin_bit, int end_bit,
                const char* tag = "sort") {
    if (n_cap == 0 || end_bit <= begin_bit) return;
    if (n_cap >= (1ull << 32)) fail(FGSS_ERR_UNSUPPORTED, "radix sort of 2^32 or more elements");
    const uint32_t ntiles = (uint32_t)((n_cap + kSortTile - 1) / kSortTile);
    std::string t(tag);
    K* k2 = c.devT<K>(t + ".k", n_cap);
    V* v2 = values ? c.devT<V>(t + ".v", n_cap) : nullptr;
    uint32_t* hist = c.devT<uint32_t>(t + ".hist", (uint64_t)256 * ntiles + 1);
    K* ka = keys;
    K* kb = k2;
    V* va = values;
    V* vb = v2;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8, passes++) {
        k_sort_hist<K><<<ntiles, kSortThreads, 0, c.stream>>>(ka, hist, n_cap, d_n, shift, ntiles);
        FGSS_LAUNCH_CK();
        exclusive_scan<uint32_t>(c, hist, hist, (uint64_t)256 * ntiles, nullptr, (uint32_t*)nullptr,
                                 (t + ".hs").c_str());
        k_sort_scatter<K, V><<<ntiles, kSortThreads, 0, c.stream>>>(ka, kb, va, vb, hist, n_cap, d_n, shift,
                                                                     ntiles);
        FGSS_LAUNCH_CK();
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (passes & 1) {
        // result sits in scratch: copy back (element count from the device when given)
        FGSS_CK(cudaMemcpyAsync(keys, ka, n_cap * sizeof(K), cudaMemcpyDeviceToDevice, c.stream));
        if (values) FGSS_CK(cudaMemcpyAsync(values, va, n_cap * sizeof(V), cudaMemcpyDeviceToDevice, c.stream));
    }
}

}  // namespace fgss
