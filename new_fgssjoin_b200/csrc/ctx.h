// ctx.h -- the library context: device, stream, a grow-only device buffer
// pool (no allocation once a workload size has been seen), cached bound
// tables, the learned cost model and the autotuner table.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

struct fgss_model;  // model.cu

namespace fgss {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// Autotuned launch shapes of the fused filter/verify kernel, per workload class.
struct TuneEntry {
    int threads = 64;      // CTA size
    int hash_log2 = 9;     // shared-memory slot table (log2)
    int regs_rt = 1024;    // resident threads per SM the register budget is sized for
    int ctas_per_sm = 0;   // persistent grid = ctas_per_sm x SMs (0 = as many as fit)
    int heavy_min_probe = 0;  // queries with a probe prefix this long take the global accumulator (0: only
                              // those beyond the fused kernel's shared-memory caps)
    float ms = 0.f;        // best time seen
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int verbose = 0;
    int num_sms = 148;
    size_t smem_optin = 227 * 1024;
    std::string last_error;
    std::string tune_path;
    std::map<std::string, DevBuf> bufs;
    std::map<std::string, DevBuf> host_bufs;  // pinned
    std::map<std::string, TuneEntry> tune;
    const TuneEntry* tune_force = nullptr;  // set by the autotuner while it times a shape
    // Buffer-name namespace of the batch-level buffers: "" normally, a graph's
    // own "g<id>." while a graph-eligible batch is recorded or captured, so no
    // later call can move a buffer a captured graph points to.
    std::string bpfx;
    struct GraphCache* graphs = nullptr;  // captured batched pipelines (api.cu)
    fgss_model* model = nullptr;
    cudaEvent_t ev[8] = {};
    bool probe_timed = false;  // ev[4]..ev[5] bracket the last fused filter+verify launch
    bool heavy_timed = false;  // ev[6]..ev[7] bracket the last global-accumulator launch

    // Device buffer `name` of at least `bytes`; grows (never shrinks) and keeps
    // its address while big enough, so repeated calls at one size allocate nothing.
    void* dev(const std::string& name, size_t bytes) {
        if (bytes == 0) bytes = 16;
        DevBuf& b = bufs[name];
        if (b.bytes < bytes) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (stream && cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
                fail(FGSS_ERR_CUDA, "buffer " + name + " would grow during a graph capture");
            if (b.p) FGSS_CK(cudaFree(b.p));
            b.p = nullptr;
            b.bytes = 0;
            size_t nb = bytes + bytes / 8 + 256;
            FGSS_CK(cudaMalloc(&b.p, nb));
            b.bytes = nb;
        }
        return b.p;
    }
    template <typename T>
    T* devT(const std::string& name, size_t count) {
        return static_cast<T*>(dev(name, count * sizeof(T)));
    }
    void* pinned(const std::string& name, size_t bytes) {
        if (bytes == 0) bytes = 16;
        DevBuf& b = host_bufs[name];
        if (b.bytes < bytes) {
            if (b.p) FGSS_CK(cudaFreeHost(b.p));
            b.p = nullptr;
            b.bytes = 0;
            size_t nb = bytes + bytes / 8 + 256;
            FGSS_CK(cudaMallocHost(&b.p, nb));
            b.bytes = nb;
        }
        return b.p;
    }
    template <typename T>
    T* pinnedT(const std::string& name, size_t count) {
        return static_cast<T*>(pinned(name, count * sizeof(T)));
    }
    void sync() { FGSS_CK(cudaStreamSynchronize(stream)); }
    // Frees every pooled device buffer whose name starts with `prefix`.
    void release_prefix(const std::string& prefix) {
        for (auto it = bufs.begin(); it != bufs.end();) {
            if (it->first.compare(0, prefix.size(), prefix) == 0) {
                if (it->second.p) cudaFree(it->second.p);
                it = bufs.erase(it);
            } else {
                ++it;
            }
        }
    }
};

}  // namespace fgss

struct fgss_ctx {
    fgss::Ctx c;
};
