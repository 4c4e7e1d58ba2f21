// common.cuh -- shared host/device helpers of libfgss (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/fgss.h"

namespace fgss {

struct Error {
    fgss_status st;
    std::string msg;
};

[[noreturn]] inline void fail(fgss_status st, const std::string& msg) { throw Error{st, msg}; }

#define FGSS_CK(x)                                                                                   \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess) {                                                                     \
            (void)cudaGetLastError();                                                                \
            ::fgss::fail(e_ == cudaErrorMemoryAllocation ? FGSS_ERR_NOMEM : FGSS_ERR_CUDA,          \
                         std::string(#x) + ": " + cudaGetErrorString(e_) + " at " + __FILE__ + ":" + \
                             std::to_string(__LINE__));                                              \
        }                                                                                            \
    } while (0)

// Kernel launches issued by this thread (read as a delta around a call).
inline unsigned long long& launch_counter() {
    static thread_local unsigned long long n = 0;
    return n;
}
#define FGSS_LAUNCH_CK()                 \
    do {                                 \
        ++::fgss::launch_counter();      \
        FGSS_CK(cudaGetLastError());     \
    } while (0)

constexpr int kWarp = 32;
constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(kFull, v, o);
        if (lane_id() >= (uint32_t)o) v += u;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024).
// `wsum` is shared scratch of 33 elements.  Returns the exclusive prefix and
// writes the block total to *total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* wsum, T* total) {
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    T inc = warp_incl_scan(v);
    if (lane == 31 || threadIdx.x == blockDim.x - 1) wsum[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T x = lane < nw ? wsum[lane] : T(0);
        T xi = warp_incl_scan(x);
        if (lane < nw) wsum[lane] = xi - x;
        if (lane == nw - 1) wsum[32] = xi;
    }
    __syncthreads();
    T r = inc - v + wsum[wid];
    *total = wsum[32];
    __syncthreads();
    return r;
}

inline unsigned grid_for(uint64_t n, unsigned per_block, unsigned cap = 1u << 30) {
    uint64_t g = (n + per_block - 1) / per_block;
    if (g == 0) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

}  // namespace fgss
