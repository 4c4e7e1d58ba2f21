// noalloc.cu -- an exclusive scan that never allocates device memory.
//
// fgss_dev_exclusive_scan_u32 takes its tile-sum scratch from the context's
// buffer pool, which calls cudaMalloc the first time a size is seen.  Some
// callers cannot allow that: a host that pre-allocates all device memory at
// start-up and forbids later allocations (its own memory cap or pool), or a
// latency-critical loop where cudaMalloc / cudaFree would stall it (cudaFree
// synchronizes the device).  fgss_dev_exclusive_scan_u32_noalloc serves them:
// its scratch is the fixed array below, so it needs neither a context nor an
// allocation, only the caller's input, output and stream.
#include <mutex>
#include <string>

#include "prims.cuh"

namespace fgss {
void set_thread_error(const std::string& msg);
}

namespace {

// Tile sums of one scan: one uint32 per 4096 input elements.  65536 slots
// (256 KiB, held on every device that loads the library until the process
// exits) bound a call to 65536 x 4096 = 268,435,456 elements.
constexpr uint64_t kNoAllocTiles = 65536;
__device__ __align__(256) uint32_t g_scan_scratch[kNoAllocTiles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// Device address of g_scan_scratch on the current device (the host-side name
// of the array is not a device address).  It is looked up again on every call
// whose stream is not capturing, so a device reset (or the primary context
// being torn down and re-created), which moves the array, never leaves a stale
// address behind; a call under stream capture takes the address of the last
// uncaptured call on this device.
uint32_t* scratch_for_current_device(cudaStream_t stream, int* err_dev) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *err_dev = dev;
        return nullptr;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    bool capturing = true;  // if the stream cannot tell, keep out of the lookup
    if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess) capturing = cs != cudaStreamCaptureStatusNone;
    else (void)cudaGetLastError();
    std::lock_guard<std::mutex> lock(g_mu);
    if (!capturing) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scan_scratch) != cudaSuccess) {
            (void)cudaGetLastError();
            *err_dev = dev;
            return nullptr;
        }
        g_scratch_addr[dev] = static_cast<uint32_t*>(p);
    }
    if (!g_scratch_addr[dev]) *err_dev = dev;
    return g_scratch_addr[dev];
}

}  // namespace

extern "C" fgss_status fgss_dev_exclusive_scan_u32_noalloc(const uint32_t* in, uint32_t* out, uint64_t n,
                                                           void* stream) {
    using namespace fgss;
    if (n == 0) return FGSS_OK;
    if (!in || !out) {
        set_thread_error("fgss_dev_exclusive_scan_u32_noalloc: null input or output");
        return FGSS_ERR_INVALID;
    }
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles > kNoAllocTiles) {
        set_thread_error("fgss_dev_exclusive_scan_u32_noalloc: n = " + std::to_string(n) +
                         " exceeds the fixed scratch limit of " + std::to_string(kNoAllocTiles * kScanTile) +
                         " elements");
        return FGSS_ERR_CAPACITY;
    }
    int dev = -1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* sums = scratch_for_current_device(s, &dev);
    if (!sums) {
        set_thread_error("fgss_dev_exclusive_scan_u32_noalloc: no scratch address on device " + std::to_string(dev) +
                         " (the first call on a device, and the first after a device reset, must not be captured)");
        return FGSS_ERR_CUDA;
    }
    // Every tile sum the later kernels read is written by k_scan_tiles first,
    // so the array's contents from an earlier call never leak into this one.
    k_scan_tiles<uint32_t><<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, out, sums, n, nullptr);
    k_scan_totals<uint32_t><<<1, 1024, 0, s>>>(sums, ntiles, n, nullptr, (uint32_t*)nullptr);
    k_scan_add<uint32_t><<<(unsigned)ntiles, kScanThreads, 0, s>>>(out, sums, n, nullptr);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_thread_error(std::string("fgss_dev_exclusive_scan_u32_noalloc: ") + cudaGetErrorString(e));
        return FGSS_ERR_CUDA;
    }
    return FGSS_OK;
}
