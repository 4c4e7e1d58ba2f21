// api.cu -- the extern "C" boundary of libfgss (include/fgss.h).  Every entry
// point catches the library's internal errors and returns a status; nothing
// here exits the process (the reference calls exit(1) on any CUDA error,
// src/util.cu:43-49).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "join.h"
#include "model.h"
#include "prims.cuh"
#include "tokenize.h"

using namespace fgss;

namespace {
thread_local std::string g_err;
}

namespace fgss {
// Message for fgss_last_error(NULL) from entry points that take no context.
void set_thread_error(const std::string& msg) { g_err = msg; }
}  // namespace fgss

namespace {

template <typename F>
fgss_status guard(fgss_ctx* ctx, F&& f) {
    try {
        f();
        if (ctx) ctx->c.last_error.clear();
        return FGSS_OK;
    } catch (const Error& e) {
        if (ctx) ctx->c.last_error = e.msg;
        g_err = e.msg;
        return e.st;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->c.last_error = "host allocation failed";
        return FGSS_ERR_NOMEM;
    } catch (...) {
        if (ctx) ctx->c.last_error = "unknown error";
        return FGSS_ERR_CUDA;
    }
}

struct PairsPriv {
    bool host_owned;
};

void fill_stats(const JoinState& J, fgss_stats* st) {
    if (!st) return;
    st->candidates = J.stats_host[SS_CANDIDATES];
    st->intersections = J.stats_host[SS_INTERSECTIONS];
    st->results = J.n_res;
    st->probe_tokens = J.stats_host[SS_PROBE];
    st->window_entries = J.stats_host[SS_WINDOW];
    st->verified = J.stats_host[SS_VERIFIED];
    st->heavy_queries = J.stats_host[SS_HEAVY];
    st->overflow_retries = J.overflow_retries;
    st->merged_tokens = J.stats_host[SS_MERGED];
    st->query_tokens = J.stats_host[SS_QTOK];
    st->predicted_candidates = J.pred_candidates;
    st->predicted_results = J.pred_results;
}

// Page-locked host blocks for the pairs handed to the caller: the device-to-host
// copies of the columns run at the link's rate and write no freshly mapped
// pages.  fgss_pairs_free gives a block back to a process-wide pool that the
// next call takes it from; the pool keeps at most kPinnedPoolBytes of free
// blocks and releases the rest.  Where page-locked memory cannot be had the
// columns are malloc'd as before.
struct PinnedPool {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;  // size -> free block
    std::map<void*, size_t> sizes;             // every block of the pool, handed out or free
    size_t free_bytes = 0;
};
constexpr size_t kPinnedPoolBytes = size_t(1) << 30;

PinnedPool& pinned_pool() {
    static PinnedPool* pool = new PinnedPool;  // never destroyed: blocks may be given back at exit
    return *pool;
}

// A block of at least `bytes` (a free one of at most twice the size, else a new
// one), or nullptr.
void* pinned_take(size_t bytes) {
    PinnedPool& P = pinned_pool();
    {
        std::lock_guard<std::mutex> lk(P.mu);
        auto it = P.free_blocks.lower_bound(bytes);
        if (it != P.free_blocks.end() && it->first <= 2 * bytes + (size_t(1) << 20)) {
            void* b = it->second;
            P.free_bytes -= it->first;
            P.free_blocks.erase(it);
            return b;
        }
    }
    void* b = nullptr;
    if (cudaHostAlloc(&b, bytes, cudaHostAllocPortable) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(P.mu);
    P.sizes[b] = bytes;
    return b;
}

// Gives a block of the pool back (true), or returns false for other memory.
bool pinned_give(void* b) {
    PinnedPool& P = pinned_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.sizes.find(b);
    if (it == P.sizes.end()) return false;
    const size_t sz = it->second;
    if (P.free_bytes + sz <= kPinnedPoolBytes) {
        P.free_blocks.emplace(sz, b);
        P.free_bytes += sz;
    } else {
        P.sizes.erase(it);
        if (cudaFreeHost(b) != cudaSuccess) (void)cudaGetLastError();
    }
    return true;
}

// Host columns of R pairs (freed by fgss_pairs_free): one page-locked block of
// six 256-byte aligned columns (priv = the block), else six malloc'd columns.
void alloc_host_pairs(fgss_pairs* out, uint64_t R) {
    const size_t col = ((R ? R : 1) * 4 + 255) & ~size_t(255);
    if (void* blk = pinned_take(6 * col)) {
        char* b = static_cast<char*>(blk);
        out->q = reinterpret_cast<uint32_t*>(b);
        out->s = reinterpret_cast<uint32_t*>(b + col);
        out->id_q = reinterpret_cast<uint32_t*>(b + 2 * col);
        out->id_s = reinterpret_cast<uint32_t*>(b + 3 * col);
        out->overlap = reinterpret_cast<uint32_t*>(b + 4 * col);
        out->sim = reinterpret_cast<float*>(b + 5 * col);
        out->priv = blk;
        return;
    }
    const size_t b = (R ? R : 1) * 4;
    out->q = (uint32_t*)malloc(b);
    out->s = (uint32_t*)malloc(b);
    out->id_q = (uint32_t*)malloc(b);
    out->id_s = (uint32_t*)malloc(b);
    out->overlap = (uint32_t*)malloc(b);
    out->sim = (float*)malloc(b);
    if (!out->q || !out->s || !out->id_q || !out->id_s || !out->overlap || !out->sim)
        fail(FGSS_ERR_NOMEM, "host allocation for pairs");
}

void export_pairs(Ctx& c, JoinState& J, const fgss_join_opts& o, fgss_pairs* out) {
    memset(out, 0, sizeof *out);
    const uint64_t R = J.n_res;
    out->n = R;
    if (o.out_on_device) {
        // hand out library buffers: copies so the context can be reused
        auto dup = [&](const void* src, size_t bytes) -> void* {
            void* p = nullptr;
            FGSS_CK(cudaMalloc(&p, bytes ? bytes : 4));
            if (bytes) FGSS_CK(cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToDevice, c.stream));
            return p;
        };
        out->q = (uint32_t*)dup(J.oq, R * 4);
        out->s = (uint32_t*)dup(J.os, R * 4);
        out->id_q = (uint32_t*)dup(J.oidq, R * 4);
        out->id_s = (uint32_t*)dup(J.oids, R * 4);
        out->overlap = (uint32_t*)dup(J.oo, R * 4);
        out->sim = (float*)dup(J.osim, R * 4);
        out->on_device = 1;
    } else {
        alloc_host_pairs(out, R);
        if (R) {
            FGSS_CK(cudaMemcpyAsync(out->q, J.oq, R * 4, cudaMemcpyDeviceToHost, c.stream));
            FGSS_CK(cudaMemcpyAsync(out->s, J.os, R * 4, cudaMemcpyDeviceToHost, c.stream));
            FGSS_CK(cudaMemcpyAsync(out->id_q, J.oidq, R * 4, cudaMemcpyDeviceToHost, c.stream));
            FGSS_CK(cudaMemcpyAsync(out->id_s, J.oids, R * 4, cudaMemcpyDeviceToHost, c.stream));
            FGSS_CK(cudaMemcpyAsync(out->overlap, J.oo, R * 4, cudaMemcpyDeviceToHost, c.stream));
            FGSS_CK(cudaMemcpyAsync(out->sim, J.osim, R * 4, cudaMemcpyDeviceToHost, c.stream));
        }
        out->on_device = 0;
    }
    if (!J.cand_host.empty() || o.want_candidates) {
        out->n_cand = J.cand_host.size() / 3;
        out->cand = (uint32_t*)malloc((J.cand_host.size() + 1) * 4);
        if (!J.cand_host.empty()) memcpy(out->cand, J.cand_host.data(), J.cand_host.size() * 4);
    }
    c.sync();
}

// Pairs of every join of a batch: host outputs through one pinned staging
// copy per column of the batch's output range, then a host copy per join.
void export_batch(Ctx& c, Batch& B, const fgss_join_opts* opts, fgss_pairs* outs) {
    const size_t nj = B.js.size();
    bool staged = nj > 1;
    for (size_t j = 0; j < nj; j++) staged &= !opts[j].out_on_device && !opts[j].want_candidates;
    if (!staged) {
        for (size_t j = 0; j < nj; j++) export_pairs(c, *B.js[j], opts[j], &outs[j]);
        return;
    }
    const uint64_t oc = B.out_cap;
    uint32_t* st = c.pinnedT<uint32_t>("b.stage", 6 * oc + 1);
    const void* cols[6] = {B.oq, B.os, B.oidq, B.oids, B.oo, B.osim};
    if (oc) {
        for (int k = 0; k < 6; k++)
            FGSS_CK(cudaMemcpyAsync(st + k * oc, cols[k], oc * 4, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    }
    for (size_t j = 0; j < nj; j++) {
        fgss_pairs* out = &outs[j];
        memset(out, 0, sizeof *out);
        const uint64_t R = B.js[j]->n_res, o = B.out_off[j];
        out->n = R;
        alloc_host_pairs(out, R);
        void* dst[6] = {out->q, out->s, out->id_q, out->id_s, out->overlap, out->sim};
        for (int k = 0; k < 6; k++) memcpy(dst[k], st + k * oc + o, R * 4);
    }
}

// Device times of a call: index build, filter+verify, output, fused launch.
struct Times {
    float idx = 0, fv = 0, out = 0, probe = 0, heavy = 0;
};

// Adds the times the events ev[0..2] (and ev[4..5], ev[6..7]) bracket, up to now.
void add_times(Ctx& c, Times& t) {
    cudaEvent_t* ev = c.ev;
    FGSS_CK(cudaEventRecord(ev[3], c.stream));
    FGSS_CK(cudaEventSynchronize(ev[3]));
    float a = 0, b = 0, d = 0, e = 0;
    FGSS_CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
    FGSS_CK(cudaEventElapsedTime(&b, ev[1], ev[2]));
    FGSS_CK(cudaEventElapsedTime(&d, ev[2], ev[3]));
    if (c.probe_timed) FGSS_CK(cudaEventElapsedTime(&e, ev[4], ev[5]));
    float hv = 0;
    if (c.heavy_timed) FGSS_CK(cudaEventElapsedTime(&hv, ev[6], ev[7]));
    c.probe_timed = false;
    c.heavy_timed = false;
    t.heavy += hv;
    t.idx += a;
    t.fv += b;
    t.out += d;
    t.probe += e;
}

void report_stats(Ctx& c, std::vector<JoinState*>& js, fgss_stats* stats, unsigned long long launches, int n,
                  const Times& t) {
    if (stats) {
        uint64_t* he = c.pinnedT<uint64_t>("h.E", (size_t)n + 1);
        bool any = false;
        for (int i = 0; i < n; i++) {
            if (js[i]->n_entries != ~0ull) continue;
            FGSS_CK(cudaMemcpyAsync(he + i, js[i]->d_e, 8, cudaMemcpyDeviceToHost, c.stream));
            any = true;
        }
        if (any) c.sync();
        for (int i = 0; i < n; i++) {
            memset(&stats[i], 0, sizeof(fgss_stats));
            fill_stats(*js[i], &stats[i]);
            stats[i].index_entries = js[i]->n_entries != ~0ull ? js[i]->n_entries : he[i];
            stats[i].ms_index = t.idx;
            stats[i].ms_filter = t.fv;
            stats[i].ms_output = t.out;
            stats[i].ms_total = t.idx + t.fv + t.out;
            stats[i].ms_probe = t.probe;
            stats[i].ms_heavy = t.heavy;
            stats[i].launches = launches;
        }
    }
    if (c.verbose)
        fprintf(stderr, "[fgss] joins=%d index %.3f ms, filter+verify %.3f ms, output %.3f ms\n", n, t.idx, t.fv,
                t.out);
}

}  // namespace

// ---------------------------------------------------------------- graphs
//
// A batched call whose inputs are all on the device is recorded eagerly the
// first time (BatchPlan) and then captured, index build included, into one
// CUDA graph under its own buffer namespace.  A later call with the same
// inputs (device pointers, sizes, thresholds, options) re-validates its input
// eagerly, replays the graph, and falls back to the eager path if any
// presized buffer overflowed.
namespace fgss {
struct GraphEntry {
    cudaGraphExec_t exec = nullptr;   // null: not captured (yet); calls run eagerly in ns
    int failed_captures = 0;
    std::string ns;
    std::vector<std::unique_ptr<JoinState>> joins;
    std::unique_ptr<Batch> batch;     // the batch the graph was captured from (its buffers)
    BatchPlan plan;
    unsigned long long launches = 0;  // kernels inside the graph
    uint64_t stamp = 0;
};

struct GraphCache {
    std::map<std::string, std::unique_ptr<GraphEntry>> entries;
    uint64_t next_id = 0, clock = 0;
};
}  // namespace fgss

namespace {

constexpr size_t kMaxGraphs = 4;
constexpr int kMaxCaptureTries = 2;  // an entry whose capture failed this often stays eager

void drop_graph(Ctx& c, std::unique_ptr<GraphEntry>& g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    c.release_prefix(g->ns);
    g.reset();
}

}  // namespace

// Drops every captured batch (after the tuned shapes or the model changed).
void fgss::clear_graphs(Ctx& c) {
    if (!c.graphs) return;
    cudaStreamSynchronize(c.stream);
    for (auto& kv : c.graphs->entries) drop_graph(c, kv.second);
    c.graphs->entries.clear();
}

namespace {

std::string graph_key(const fgss_sets_view* sets, const fgss_join_opts* opts, int n) {
    std::string k;
    char buf[256];
    for (int i = 0; i < n; i++) {
        uint32_t tb;
        memcpy(&tb, &opts[i].threshold, 4);
        snprintf(buf, sizeof buf, "%p,%p,%p,%p,%llu,%llu,%u|%u,%d,%d,%llu,%llu,%llu,%d;", (const void*)sets[i].id,
                 (const void*)sets[i].pos, (const void*)sets[i].len, (const void*)sets[i].tokens,
                 (unsigned long long)sets[i].n_sets, (unsigned long long)sets[i].n_tokens, sets[i].n_terms, tb,
                 opts[i].bounds, opts[i].use_model, (unsigned long long)opts[i].result_capacity,
                 (unsigned long long)opts[i].query_begin, (unsigned long long)opts[i].query_end, opts[i].filter);
        k += buf;
    }
    return k;
}

// Splits a batched call into groups of consecutive joins whose batch-level
// per-record offsets (32-bit) and result sort keys (64-bit) fit; nearly
// every batch is one group.
std::vector<std::pair<int, int>> batch_groups(const fgss_sets_view* sets, int n) {
    std::vector<std::pair<int, int>> g;
    int b = 0;
    uint64_t T = 0, R = 0, nmax = 0;
    for (int i = 0; i < n; i++) {
        const uint64_t t = sets[i].n_tokens, r = sets[i].n_sets, nm = std::max(nmax, r);
        const bool fits = T + t < (1ull << 31) && R + r < (1ull << 31) && 2 * bits_for(nm) + bits_for(i - b + 1) <= 64;
        if (!fits && i > b) {
            g.push_back({b, i});
            b = i;
            T = R = nmax = 0;
        }
        T += t;
        R += r;
        nmax = std::max(nmax, r);
    }
    g.push_back({b, n});
    return g;
}

// Replays a captured batch; false when its presized buffers are too small for
// this call's data (the caller then runs the exact eager path).
bool replay_graph(Ctx& c, GraphEntry& g, const fgss_sets_view* sets, const fgss_join_opts* opts, int n,
                  fgss_pairs* outs, fgss_stats* stats) {
    c.bpfx = g.ns;
    c.probe_timed = false;
    c.heavy_timed = false;
    std::vector<JoinState*> v;
    for (auto& j : g.joins) v.push_back(j.get());
    Batch& B = *g.batch;
    FGSS_CK(cudaEventRecord(c.ev[0], c.stream));
    // validation, fresh counters and the index and probe totals; the graph
    // holds every later stage
    batch_prep(c, B, v, sets, opts);
    if (B.E > g.plan.E_cap || B.P > g.plan.P_cap) {
        c.bpfx.clear();
        return false;
    }
    FGSS_CK(cudaEventRecord(c.ev[1], c.stream));
    FGSS_CK(cudaGraphLaunch(g.exec, c.stream));
    launch_counter() += g.launches;
    c.probe_timed = true;
    c.heavy_timed = g.plan.heavy_slots > 0;
    FGSS_CK(cudaEventRecord(c.ev[2], c.stream));
    uint32_t* h = c.pinnedT<uint32_t>(g.ns + "h.st", 8 * (size_t)n);
    FGSS_CK(cudaMemcpyAsync(h, B.status, 32 * (size_t)n, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    for (int i = 0; i < n; i++) {
        const uint32_t bad = ST_RES_OVERFLOW | ST_HEAVY_OVERFLOW | ST_HASH_FULL;
        if ((h[8 * i] & bad) || h[8 * i + 3] > g.plan.res_cap[i]) {
            c.bpfx.clear();
            return false;
        }
    }
    batch_finish_status(c, B);
    c.bpfx.clear();
    for (int i = 0; i < n; i++) v[i]->overflow_retries = 0;
    export_batch(c, B, opts, outs);
    Times t;
    add_times(c, t);
    report_stats(c, v, stats, g.launches, n, t);
    return true;
}

void run_joins(Ctx& c, const fgss_sets_view* sets, const fgss_join_opts* opts, int n, fgss_pairs* outs,
               fgss_stats* stats) {
    if (n <= 0) return;
    if (!sets || !opts || !outs) fail(FGSS_ERR_INVALID, "null argument");
    bool batched = false;
    for (int i = 0; i < n; i++) batched |= opts[i].method == FGSS_METHOD_BATCHED;
    if (batched && opts[0].want_candidates) fail(FGSS_ERR_INVALID, "want_candidates needs the plain method");
    const std::vector<std::pair<int, int>> groups =
        batched ? batch_groups(sets, n) : std::vector<std::pair<int, int>>{{0, n}};
    bool graphable = batched && !c.tune_force && c.graphs && groups.size() == 1;
    for (int i = 0; i < n; i++) graphable &= sets[i].on_device != 0 && !opts[i].no_graph;
    std::string gkey;
    std::unique_ptr<GraphEntry> g;
    if (graphable) {
        gkey = graph_key(sets, opts, n);
        auto it = c.graphs->entries.find(gkey);
        if (it != c.graphs->entries.end()) {
            it->second->stamp = ++c.graphs->clock;
            if (it->second->exec) {
                bool ok = false;
                try {
                    ok = replay_graph(c, *it->second, sets, opts, n, outs, stats);
                } catch (...) {
                    c.bpfx.clear();
                    throw;
                }
                if (ok) return;
                // its plan no longer fits the data: record a new one in the same buffers
                cudaGraphExecDestroy(it->second->exec);
                it->second->exec = nullptr;
            }
            g = std::move(it->second);
            c.graphs->entries.erase(it);
        }
        if (!g) {
            g.reset(new GraphEntry());
            g->ns = "g" + std::to_string(c.graphs->next_id++) + ".";
        }
        c.bpfx = g->ns;
    }
    std::vector<std::unique_ptr<JoinState>> js(n);
    std::vector<JoinState*> jv(n);
    for (int i = 0; i < n; i++) {
        js[i].reset(new JoinState());
        js[i]->slot = i;
        if (g) js[i]->ns = g->ns;
        jv[i] = js[i].get();
    }
    cudaEvent_t* ev = c.ev;
    const unsigned long long launches0 = launch_counter();
    c.probe_timed = false;
    c.heavy_timed = false;
    Times times;
    BatchPlan plan;
    std::unique_ptr<Batch> Bp(new Batch());
    try {
        if (!batched) {
            FGSS_CK(cudaEventRecord(ev[0], c.stream));
            for (int i = 0; i < n; i++) {
                fgss_sets_view v = sets[i];
                if (!v.on_device) {
                    // the same host arrays as an earlier join of the batch: copied to the device once
                    for (int j = 0; j < i; j++) {
                        const fgss_sets_view& w = sets[j];
                        if (!w.on_device && w.id == v.id && w.pos == v.pos && w.len == v.len &&
                            w.tokens == v.tokens && w.n_sets == v.n_sets && w.n_tokens == v.n_tokens) {
                            v = js[j]->in;
                            v.n_terms = sets[i].n_terms;
                            break;
                        }
                    }
                }
                join_setup(c, *js[i], v, opts[i], i, false);
            }
            c.sync();  // one wait for the whole batch's input validation
            for (int i = 0; i < n; i++) join_check_input(c, *js[i]);
            for (int i = 0; i < n; i++) join_index(c, *js[i]);
            FGSS_CK(cudaEventRecord(ev[1], c.stream));
            for (int i = 0; i < n; i++) join_plain_filter_verify(c, *js[i], opts[i].want_candidates != 0);
            FGSS_CK(cudaEventRecord(ev[2], c.stream));
            for (int i = 0; i < n; i++) {
                join_finish_status(c, *js[i]);
                export_pairs(c, *js[i], opts[i], &outs[i]);
            }
            add_times(c, times);
        } else {
            for (const auto& gr : groups) {
                Batch& B = *Bp;
                std::vector<JoinState*> v;
                for (int i = gr.first; i < gr.second; i++) v.push_back(jv[i]);
                FGSS_CK(cudaEventRecord(ev[0], c.stream));
                batch_prep(c, B, v, sets + gr.first, opts + gr.first);
                plan.E_cap = B.E;
                plan.P_cap = B.P;
                batch_index(c, B, B.E);
                FGSS_CK(cudaEventRecord(ev[1], c.stream));
                batched_filter_verify(c, B, opts[gr.first].use_model != 0, g ? &plan : nullptr);
                FGSS_CK(cudaEventRecord(ev[2], c.stream));
                batch_finish_status(c, B);
                export_batch(c, B, opts + gr.first, outs + gr.first);
                add_times(c, times);
            }
        }
        report_stats(c, jv, stats, launch_counter() - launches0, n, times);
        if (g && g->failed_captures < kMaxCaptureTries) {
            // capture the same batch (index build included) for later calls
            plan.capture = true;
            const unsigned long long l0 = launch_counter();
            cudaGraph_t graph = nullptr;
            FGSS_CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
            bool captured = true;
            try {
                batch_index(c, *Bp, plan.E_cap);
                batched_filter_verify(c, *Bp, opts[0].use_model != 0, &plan);
            } catch (const Error& e) {
                captured = false;  // this call's results stand; later calls run eagerly
                if (c.verbose) fprintf(stderr, "[fgss] graph capture skipped: %s\n", e.msg.c_str());
            }
            const cudaError_t ec = cudaStreamEndCapture(c.stream, &graph);
            (void)cudaGetLastError();
            if (captured && ec == cudaSuccess && graph) {
                captured = cudaGraphInstantiate(&g->exec, graph, 0) == cudaSuccess;
                (void)cudaGetLastError();
            } else {
                captured = false;
            }
            if (graph) cudaGraphDestroy(graph);
            g->launches = launch_counter() - l0;
            launch_counter() = l0;  // captured, not launched
            if (captured) {
                g->joins = std::move(js);
                g->batch = std::move(Bp);
                g->plan = plan;
            } else {
                g->failed_captures++;  // later calls run eagerly in the same buffers
            }
        }
        if (g) {
            // keep the entry (and its buffers) for the next call with these inputs
            g->stamp = ++c.graphs->clock;
            if (c.graphs->entries.size() >= kMaxGraphs) {
                auto oldest = c.graphs->entries.begin();
                for (auto it = c.graphs->entries.begin(); it != c.graphs->entries.end(); ++it)
                    if (it->second->stamp < oldest->second->stamp) oldest = it;
                drop_graph(c, oldest->second);
                c.graphs->entries.erase(oldest);
            }
            c.graphs->entries[gkey] = std::move(g);
        }
    } catch (...) {
        c.bpfx.clear();
        if (g) {
            cudaStreamSynchronize(c.stream);
            c.release_prefix(g->ns);
        }
        throw;
    }
    c.bpfx.clear();
}

}  // namespace

extern "C" {

int fgss_version(void) { return FGSS_VERSION_MAJOR * 100 + FGSS_VERSION_MINOR; }

const char* fgss_strerror(fgss_status st) {
    switch (st) {
        case FGSS_OK: return "ok";
        case FGSS_ERR_INVALID: return "invalid argument";
        case FGSS_ERR_CUDA: return "CUDA error";
        case FGSS_ERR_NOMEM: return "out of memory";
        case FGSS_ERR_FORMAT: return "malformed input";
        case FGSS_ERR_IO: return "I/O error";
        case FGSS_ERR_UNSUPPORTED: return "unsupported input";
        case FGSS_ERR_TIMEOUT: return "device wait timed out";
        case FGSS_ERR_CAPACITY: return "buffer too small";
    }
    return "unknown status";
}

const char* fgss_last_error(const fgss_ctx* ctx) { return ctx ? ctx->c.last_error.c_str() : g_err.c_str(); }

void fgss_options_default(fgss_options* o) {
    if (!o) return;
    memset(o, 0, sizeof *o);
}

void fgss_join_opts_default(fgss_join_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->threshold = 0.9f;
    o->bounds = FGSS_BOUNDS_REFERENCE;
    o->method = FGSS_METHOD_PLAIN;
}

void fgss_tok_opts_default(fgss_tok_opts* o) {
    if (!o) return;
    o->q = 3;
    o->mode = FGSS_TOK_QGRAM;
    o->pad = 0;
    o->pad_char = 1;
    o->suffix = 1;
    o->lower = 1;
}

fgss_status fgss_create(fgss_ctx** out, const fgss_options* opt) {
    if (!out) return FGSS_ERR_INVALID;
    *out = nullptr;
    fgss_ctx* ctx = new (std::nothrow) fgss_ctx();
    if (!ctx) return FGSS_ERR_NOMEM;
    fgss_status st = guard(ctx, [&] {
        fgss_options o;
        fgss_options_default(&o);
        if (opt) o = *opt;
        Ctx& c = ctx->c;
        int ndev = 0;
        FGSS_CK(cudaGetDeviceCount(&ndev));
        if (o.device < 0 || o.device >= ndev) fail(FGSS_ERR_INVALID, "no such CUDA device");
        c.device = o.device;
        FGSS_CK(cudaSetDevice(c.device));
        cudaDeviceProp prop;
        FGSS_CK(cudaGetDeviceProperties(&prop, c.device));
        if (prop.major != 10) fail(FGSS_ERR_UNSUPPORTED, "libfgss is built for sm_100a (B200) only");
        c.num_sms = prop.multiProcessorCount;
        c.smem_optin = prop.sharedMemPerBlockOptin;
        c.verbose = o.verbose;
        if (o.tune_cache_path) c.tune_path = o.tune_cache_path;
        if (o.stream) {
            c.stream = (cudaStream_t)o.stream;
            c.own_stream = false;
        } else {
            FGSS_CK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
            c.own_stream = true;
        }
        for (auto& e : c.ev) FGSS_CK(cudaEventCreate(&e));
        tune_load(c);
        c.graphs = new GraphCache();
    });
    if (st != FGSS_OK) {
        g_err = ctx->c.last_error;
        delete ctx;
        return st;
    }
    *out = ctx;
    return FGSS_OK;
}

void fgss_destroy(fgss_ctx* ctx) {
    if (!ctx) return;
    Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    clear_graphs(c);
    delete c.graphs;
    c.graphs = nullptr;
    for (auto& kv : c.bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    for (auto& kv : c.host_bufs)
        if (kv.second.p) cudaFreeHost(kv.second.p);
    for (auto& e : c.ev)
        if (e) cudaEventDestroy(e);
    if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
    delete c.model;
    delete ctx;
}

fgss_sets_view fgss_sets_view_of(const fgss_sets* s) {
    fgss_sets_view v;
    memset(&v, 0, sizeof v);
    if (!s) return v;
    v.id = s->id;
    v.pos = s->pos;
    v.len = s->len;
    v.tokens = s->tokens;
    v.n_sets = s->n_sets;
    v.n_tokens = s->n_tokens;
    v.n_terms = s->n_terms;
    v.on_device = 0;
    return v;
}

void fgss_sets_free(fgss_sets* s) {
    if (!s) return;
    free(s->id);
    free(s->pos);
    free(s->len);
    free(s->tokens);
    free(s->loc);
    memset(s, 0, sizeof *s);
}

fgss_status fgss_tokenize(fgss_ctx* ctx, const char* text, uint64_t n_bytes, const fgss_tok_opts* opts,
                          fgss_sets* out) {
    if (!ctx || !out || (!text && n_bytes)) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        fgss_tok_opts o;
        fgss_tok_opts_default(&o);
        if (opts) o = *opts;
        TokParams p{o.q, o.mode, o.pad, o.pad_char, o.suffix, o.lower};
        FGSS_CK(cudaSetDevice(ctx->c.device));
        try {
            tokenize_device(ctx->c, text, n_bytes, p, out);
        } catch (...) {
            fgss_sets_free(out);
            throw;
        }
    });
}

fgss_status fgss_tokenize_dual(fgss_ctx* ctx, const char* text_r, uint64_t n_r, const char* text_s, uint64_t n_s,
                               const fgss_tok_opts* opts, fgss_sets* out_r, fgss_sets* out_s) {
    if (!ctx || !out_r || !out_s || (!text_r && n_r) || (!text_s && n_s)) return FGSS_ERR_INVALID;
    memset(out_r, 0, sizeof *out_r);
    memset(out_s, 0, sizeof *out_s);
    return guard(ctx, [&] {
        fgss_tok_opts o;
        fgss_tok_opts_default(&o);
        if (opts) o = *opts;
        TokParams p{o.q, o.mode, o.pad, o.pad_char, o.suffix, o.lower};
        FGSS_CK(cudaSetDevice(ctx->c.device));
        // one text: R's lines, then S's; record ids count the non-empty lines
        std::string text(text_r ? text_r : "", n_r);
        uint32_t nr_lines = 0;
        for (uint64_t i = 0; i < n_r;) {
            uint64_t e = i;
            while (e < n_r && text_r[e] != '\n') e++;
            if (e > i) nr_lines++;
            i = e + 1;
        }
        if (n_r && text_r[n_r - 1] != '\n') text.push_back('\n');
        if (n_s) text.append(text_s, n_s);
        fgss_sets all;
        memset(&all, 0, sizeof all);
        try {
            tokenize_device(ctx->c, text.data(), text.size(), p, &all);
            fgss_sets* outs[2] = {out_r, out_s};
            uint64_t cnt[2] = {0, 0}, tok[2] = {0, 0};
            for (uint64_t i = 0; i < all.n_sets; i++) {
                const int sd = all.id[i] > nr_lines;
                cnt[sd]++;
                tok[sd] += all.len[i];
            }
            for (int sd = 0; sd < 2; sd++) {
                fgss_sets& d = *outs[sd];
                d.n_sets = cnt[sd];
                d.n_tokens = tok[sd];
                d.n_terms = all.n_terms;
                const size_t nb = (cnt[sd] ? cnt[sd] : 1) * 4, tb = (tok[sd] ? tok[sd] : 1) * 4;
                d.id = (uint32_t*)malloc(nb);
                d.pos = (uint32_t*)malloc(nb);
                d.len = (uint32_t*)malloc(nb);
                d.tokens = (uint32_t*)malloc(tb);
                d.loc = all.loc ? (uint32_t*)malloc(tb) : nullptr;
                if (!d.id || !d.pos || !d.len || !d.tokens || (all.loc && !d.loc))
                    fail(FGSS_ERR_NOMEM, "host allocation for token sets");
            }
            uint64_t at[2] = {0, 0}, ti[2] = {0, 0};
            for (uint64_t i = 0; i < all.n_sets; i++) {
                const int sd = all.id[i] > nr_lines;
                fgss_sets& d = *outs[sd];
                const uint64_t k = at[sd]++, l = all.len[i];
                d.id[k] = sd ? all.id[i] - nr_lines : all.id[i];
                d.pos[k] = (uint32_t)ti[sd];
                d.len[k] = (uint32_t)l;
                memcpy(d.tokens + ti[sd], all.tokens + all.pos[i], l * 4);
                if (d.loc) memcpy(d.loc + ti[sd], all.loc + all.pos[i], l * 4);
                d.max_len = std::max<uint32_t>(d.max_len, (uint32_t)l);
                ti[sd] += l;
            }
        } catch (...) {
            fgss_sets_free(&all);
            fgss_sets_free(out_r);
            fgss_sets_free(out_s);
            throw;
        }
        fgss_sets_free(&all);
    });
}

fgss_status fgss_rsjoin(fgss_ctx* ctx, const fgss_sets_view* r, const fgss_sets_view* s, const fgss_join_opts* opts,
                        fgss_pairs* out, fgss_stats* stats) {
    if (!ctx || !r || !s || !opts || !out) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        if (opts->want_candidates) fail(FGSS_ERR_INVALID, "want_candidates is for self-joins");
        if (opts->query_end > opts->query_begin) fail(FGSS_ERR_INVALID, "query ranges are for self-joins");
        cudaEvent_t* ev = c.ev;
        const unsigned long long launches0 = launch_counter();
        c.probe_timed = false;
        c.heavy_timed = false;
        FGSS_CK(cudaEventRecord(ev[0], c.stream));
        const RsInput u = rs_union(c, *r, *s);
        JoinState J;
        J.ns = "rs.";
        J.side = u.side;
        std::vector<JoinState*> v{&J};
        Batch B;
        if (opts->method == FGSS_METHOD_BATCHED) {
            batch_prep(c, B, v, &u.view, opts);
            batch_index(c, B, B.E);
            FGSS_CK(cudaEventRecord(ev[1], c.stream));
            batched_filter_verify(c, B, opts->use_model != 0, nullptr);
            FGSS_CK(cudaEventRecord(ev[2], c.stream));
            batch_finish_status(c, B);
        } else {
            join_setup(c, J, u.view, *opts, 0);
            join_index(c, J);
            FGSS_CK(cudaEventRecord(ev[1], c.stream));
            join_plain_filter_verify(c, J, false);
            FGSS_CK(cudaEventRecord(ev[2], c.stream));
            join_finish_status(c, J);
        }
        rs_output(c, J, u);
        export_pairs(c, J, *opts, out);
        Times t;
        add_times(c, t);
        report_stats(c, v, stats, launch_counter() - launches0, 1, t);
    });
}

fgss_status fgss_selfjoin(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts, fgss_pairs* out,
                          fgss_stats* stats) {
    if (!ctx || !sets || !opts || !out) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        FGSS_CK(cudaSetDevice(ctx->c.device));
        run_joins(ctx->c, sets, opts, 1, out, stats);
    });
}

fgss_status fgss_selfjoin_batch(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts, int n,
                                fgss_pairs* outs, fgss_stats* stats) {
    if (!ctx || !sets || !opts || !outs || n < 0) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        FGSS_CK(cudaSetDevice(ctx->c.device));
        run_joins(ctx->c, sets, opts, n, outs, stats);
    });
}

void fgss_pairs_free(fgss_pairs* p) {
    if (!p) return;
    if (!p->on_device && p->priv && pinned_give(p->priv)) {
        // the columns were one block of the page-locked pool
    } else if (p->on_device) {
        cudaFree(p->q);
        cudaFree(p->s);
        cudaFree(p->id_q);
        cudaFree(p->id_s);
        cudaFree(p->overlap);
        cudaFree(p->sim);
    } else {
        free(p->q);
        free(p->s);
        free(p->id_q);
        free(p->id_s);
        free(p->overlap);
        free(p->sim);
    }
    free(p->cand);
    memset(p, 0, sizeof *p);
}

fgss_status fgss_pairs_print(const fgss_pairs* p, void* file) {
    if (!p) return FGSS_ERR_INVALID;
    if (p->on_device) return FGSS_ERR_INVALID;
    FILE* f = file ? (FILE*)file : stdout;
    for (uint64_t i = 0; i < p->n; i++)
        fprintf(f, "%d %d %f\n", (int)p->id_q[i], (int)p->id_s[i], (double)p->sim[i]);  // block.cu:193
    return FGSS_OK;
}

fgss_status fgss_selfjoin_to_file(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts,
                                  const char* path, int format, int n_shards, fgss_stats* stats) {
    if (!ctx || !sets || !opts || !path || n_shards < 1 || (format != FGSS_OUT_TEXT && format != FGSS_OUT_BINARY))
        return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        if (opts->query_end > opts->query_begin) fail(FGSS_ERR_INVALID, "the shards cover every query");
        if (opts->want_candidates || opts->out_on_device) fail(FGSS_ERR_INVALID, "pairs go to the file");
        const uint64_t n = sets->n_sets;
        // the inputs go to the device once; every shard joins against them
        fgss_sets_view v = *sets;
        std::vector<uint32_t> len(n);
        if (!v.on_device) {
            uint32_t* pos = c.devT<uint32_t>("wf.pos", n + 1);
            uint32_t* ln = c.devT<uint32_t>("wf.len", n + 1);
            uint32_t* tok = c.devT<uint32_t>("wf.tok", v.n_tokens + 1);
            uint32_t* id = v.id ? c.devT<uint32_t>("wf.id", n + 1) : nullptr;
            if (n) {
                if (!v.pos || !v.len) fail(FGSS_ERR_INVALID, "null record arrays");
                FGSS_CK(cudaMemcpyAsync(pos, v.pos, n * 4, cudaMemcpyHostToDevice, c.stream));
                FGSS_CK(cudaMemcpyAsync(ln, v.len, n * 4, cudaMemcpyHostToDevice, c.stream));
                if (id) FGSS_CK(cudaMemcpyAsync(id, v.id, n * 4, cudaMemcpyHostToDevice, c.stream));
                memcpy(len.data(), v.len, n * 4);
            }
            if (v.n_tokens) {
                if (!v.tokens) fail(FGSS_ERR_INVALID, "null token array");
                FGSS_CK(cudaMemcpyAsync(tok, v.tokens, v.n_tokens * 4, cudaMemcpyHostToDevice, c.stream));
            }
            v.pos = pos;
            v.len = ln;
            v.tokens = tok;
            v.id = id;
            v.on_device = 1;
        } else if (n) {
            FGSS_CK(cudaMemcpyAsync(len.data(), v.len, n * 4, cudaMemcpyDeviceToHost, c.stream));
        }
        c.sync();
        // contiguous query ranges of about equal work (candidates grow with size^2)
        std::vector<uint64_t> cut{0};
        {
            double tot = 0;
            for (uint64_t i = 0; i < n; i++) tot += (double)len[i] * len[i] + 1.0;
            double acc = 0;
            uint64_t i = 0;
            for (int k = 1; k < n_shards; k++) {
                const double target = tot * k / n_shards;
                while (i < n && acc + (double)len[i] * len[i] + 1.0 <= target) acc += (double)len[i] * len[i] + 1.0, i++;
                cut.push_back(std::max(cut.back(), i));
            }
            cut.push_back(n);
        }
        FILE* f = fopen(path, format == FGSS_OUT_BINARY ? "wb" : "w");
        if (!f) fail(FGSS_ERR_IO, std::string("cannot open ") + path);
        // writer thread: formats and writes one shard while the GPU joins the next;
        // at most two shards wait in host memory
        std::mutex mu;
        std::condition_variable cv;
        std::deque<fgss_pairs> queue;
        bool closed = false, werr = false;
        std::thread writer([&] {
            std::vector<char> buf(1 << 20);
            size_t used = 0;
            auto flush = [&] {
                if (used && fwrite(buf.data(), 1, used, f) != used) werr = true;
                used = 0;
            };
            for (;;) {
                fgss_pairs p;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return closed || !queue.empty(); });
                    if (queue.empty()) break;
                    p = queue.front();
                    queue.pop_front();
                }
                cv.notify_all();
                for (uint64_t i = 0; i < p.n; i++) {
                    if (used + 64 > buf.size()) flush();
                    if (format == FGSS_OUT_TEXT) {
                        // the reference's line (block.cu:193)
                        used += (size_t)snprintf(buf.data() + used, 64, "%d %d %f\n", (int)p.id_q[i], (int)p.id_s[i],
                                                 (double)p.sim[i]);
                    } else {
                        memcpy(buf.data() + used, &p.id_q[i], 4);
                        memcpy(buf.data() + used + 4, &p.id_s[i], 4);
                        memcpy(buf.data() + used + 8, &p.sim[i], 4);
                        used += 12;
                    }
                }
                fgss_pairs_free(&p);
            }
            flush();
        });
        auto finish = [&] {
            {
                std::lock_guard<std::mutex> lk(mu);
                closed = true;
            }
            cv.notify_all();
            writer.join();
            for (auto& p : queue) fgss_pairs_free(&p);
            queue.clear();
        };
        fgss_stats total;
        memset(&total, 0, sizeof total);
        try {
            for (int k = 0; k < n_shards; k++) {
                if (cut[k + 1] == cut[k]) continue;
                fgss_join_opts o = *opts;
                o.query_begin = cut[k];
                o.query_end = cut[k + 1];
                o.no_graph = 1;  // shards differ only in their query range: one set of buffers
                fgss_pairs p;
                fgss_stats st;
                run_joins(c, &v, &o, 1, &p, &st);
                total.candidates += st.candidates;
                total.intersections += st.intersections;
                total.results += st.results;
                total.index_entries = st.index_entries;
                total.probe_tokens += st.probe_tokens;
                total.window_entries += st.window_entries;
                total.verified += st.verified;
                total.heavy_queries += st.heavy_queries;
                total.overflow_retries += st.overflow_retries;
                total.ms_total += st.ms_total;
                total.ms_index += st.ms_index;
                total.ms_filter += st.ms_filter;
                total.ms_verify += st.ms_verify;
                total.ms_output += st.ms_output;
                total.ms_probe += st.ms_probe;
                total.merged_tokens += st.merged_tokens;
                total.query_tokens += st.query_tokens;
                total.launches += st.launches;
                total.predicted_candidates += st.predicted_candidates;
                total.predicted_results += st.predicted_results;
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return queue.size() < 2; });
                queue.push_back(p);
                lk.unlock();
                cv.notify_all();
            }
        } catch (...) {
            finish();
            fclose(f);
            throw;
        }
        finish();
        if (fclose(f) != 0) werr = true;
        if (werr) fail(FGSS_ERR_IO, std::string("write failed: ") + path);
        if (stats) *stats = total;
    });
}

fgss_status fgss_autotune(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts, int reps,
                          fgss_tune_result* best) {
    if (!ctx || !sets || !opts || reps <= 0) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        fgss_join_opts o = *opts;
        o.method = FGSS_METHOD_BATCHED;
        o.want_candidates = 0;
        o.out_on_device = 1;
        o.filter = FGSS_FILTER_AUTO;
        const std::string key = tune_key(sets->n_sets, sets->n_tokens, o.threshold);
        TuneEntry win;
        win.ms = 1e30f;
        // every fused-kernel shape, then every query on the global accumulator
        for (int i = 0; i <= kNumFusedShapes; i++) {
            TuneEntry te = filter_entry(FGSS_FILTER_GLOBAL);
            if (i < kNumFusedShapes) {
                te.threads = kFusedShapes[i][0];
                te.hash_log2 = kFusedShapes[i][1];
                te.regs_rt = kFusedShapes[i][2];
                te.heavy_min_probe = 0;
            }
            te.ctas_per_sm = 0;
            c.tune_force = &te;
            float bestms = 1e30f;
            for (int r = 0; r < reps; r++) {
                fgss_pairs p;
                fgss_stats st;
                try {
                    run_joins(c, sets, &o, 1, &p, &st);
                } catch (...) {
                    c.tune_force = nullptr;
                    throw;
                }
                fgss_pairs_free(&p);
                bestms = std::min(bestms, st.ms_filter);
            }
            c.tune_force = nullptr;
            if (c.verbose)
                fprintf(stderr, "[fgss] autotune %s: threads %d hash_log2 %d regs_rt %d global %d -> %.3f ms\n",
                        key.c_str(), te.threads, te.hash_log2, te.regs_rt, te.heavy_min_probe, bestms);
            if (bestms < win.ms) {
                win = te;
                win.ms = bestms;
            }
        }
        c.tune[key] = win;
        tune_save(c);
        clear_graphs(c);  // captured batches used the previous shapes
        if (best) {
            best->threads = win.threads;
            best->hash_log2 = win.hash_log2;
            best->regs_rt = win.regs_rt;
            best->ctas_per_sm = win.ctas_per_sm;
            best->ms = win.ms;
            snprintf(best->key, sizeof best->key, "%s", key.c_str());
            best->filter = filter_of(win);
        }
    });
}

fgss_status fgss_bounds_table(float threshold, int bounds, uint32_t max_len, uint16_t* probe, uint16_t* index,
                              uint32_t* min_size, uint32_t* max_size, uint32_t* need) {
    if (max_len > kMaxLen) return FGSS_ERR_UNSUPPORTED;
    if (!(threshold > 0.0f && threshold < 1.0f) || (bounds != 0 && bounds != 1)) return FGSS_ERR_INVALID;
    BoundTables b;
    compute_bounds(threshold, bounds, b);
    for (uint32_t n = 0; n <= max_len; n++) {
        if (probe) probe[n] = b.probe[n];
        if (index) index[n] = b.index[n];
        if (min_size) min_size[n] = b.minsz[n];
        if (max_size) max_size[n] = b.maxsz[n];
    }
    if (need)
        for (uint32_t S = 0; S <= 2 * max_len; S++) need[S] = b.need[S];
    return FGSS_OK;
}

fgss_status fgss_query_costs(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts,
                             uint64_t* costs) {
    if (!ctx || !sets || !opts || (!costs && sets->n_sets)) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        fgss_join_opts o = *opts;
        o.query_begin = o.query_end = 0;  // every query gets its estimate
        JoinState J;
        std::vector<JoinState*> v{&J};
        Batch B;
        batch_prep(c, B, v, sets, &o);
        batch_index(c, B, B.E);
        batch_query_costs(c, B, o.use_model != 0, costs);
    });
}

fgss_status fgss_overlap_table(float threshold, int bounds, uint32_t max_sum, uint32_t* cand_min,
                               uint32_t* inter_min) {
    if (max_sum > 2 * kMaxLen) return FGSS_ERR_UNSUPPORTED;
    if (!(threshold > 0.0f && threshold < 1.0f) || (bounds != 0 && bounds != 1)) return FGSS_ERR_INVALID;
    BoundTables b;
    compute_bounds(threshold, bounds, b);
    for (uint32_t S = 0; S <= max_sum; S++) {
        if (cand_min) cand_min[S] = b.cand_min[S];
        if (inter_min) inter_min[S] = b.inter_min[S];
    }
    return FGSS_OK;
}

fgss_status fgss_dev_exclusive_scan_u32(fgss_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n) {
    if (!ctx || (n && (!in || !out))) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        FGSS_CK(cudaSetDevice(ctx->c.device));
        if (n) exclusive_scan<uint32_t>(ctx->c, in, out, n, nullptr, (uint32_t*)nullptr, "api.scan");
        ctx->c.sync();
    });
}

fgss_status fgss_dev_sort_pairs_u64(fgss_ctx* ctx, uint64_t* keys, uint32_t* values, uint64_t n, int begin_bit,
                                    int end_bit) {
    if (!ctx || (n && !keys) || begin_bit < 0 || end_bit > 64 || begin_bit > end_bit) return FGSS_ERR_INVALID;
    return guard(ctx, [&] {
        FGSS_CK(cudaSetDevice(ctx->c.device));
        if (n) radix_sort<uint64_t, uint32_t>(ctx->c, keys, values, n, nullptr, begin_bit, end_bit, "api.sort");
        ctx->c.sync();
    });
}

}  // extern "C"
