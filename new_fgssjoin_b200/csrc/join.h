// join.h -- host driver of the self-join (plain and batched methods).
#pragma once

#include <vector>

#include "bounds.h"
#include "ctx.h"
#include "join_kernels.cuh"
#include "tiles.cuh"

namespace fgss {

// Device tables of one threshold (cached in the context per (t, mode)).
struct DevBounds {
    uint16_t* probe;
    uint16_t* index;
    uint32_t* minsz;
    uint32_t* maxsz;
    uint32_t* lmin;
    uint32_t* cand_min;
    uint32_t* inter_min;
    uint32_t* need;
    uint4* smin;  // per length sum: (cand_min, inter_min, need, 0)
};
DevBounds device_bounds(Ctx& c, float t, int mode);

// Per-query features of the learned cost model (one row per record).
constexpr int kFeat = 8;

int bits_for(uint64_t v);  // bits needed to hold values < v (at least 1)

// Everything one join keeps on the device between stages.
struct JoinState {
    int slot = 0;              // buffer-name prefix (joins of a batch use different slots)
    fgss_sets_view in{};       // device view
    const uint32_t* id = nullptr;
    float t = 0.f;
    int bounds = 0;
    int filter = 0;            // FGSS_FILTER_* (batched method)
    DevBounds lut{};
    JoinArgs args{};
    JoinArgs* d_args = nullptr;
    uint32_t* status = nullptr;
    unsigned long long* stats = nullptr;
    uint64_t* d_e = nullptr;   // index entries (u64 copy of the scan total)
    uint32_t* icnt = nullptr;
    uint32_t* pcnt = nullptr;
    uint32_t* maxlen = nullptr;
    int term_bits = 1;
    // outputs (device)
    uint64_t* d_nres = nullptr;
    uint32_t *oq = nullptr, *os = nullptr, *oidq = nullptr, *oids = nullptr, *oo = nullptr;
    float* osim = nullptr;
    uint64_t n_res = 0;
    uint64_t n_entries = ~0ull;  // index entries once read back (batched method)
    uint64_t res_cap_hint = 0;   // exact result count after an overflow
    uint64_t res_cap_user = 0;   // caller's result capacity (fgss_join_opts.result_capacity)
    uint32_t overflow_retries = 0;
    uint32_t status_host = 0;
    unsigned long long stats_host[SS_N] = {};
    std::vector<uint32_t> cand_host;  // (q, s, partial) triples when requested
    uint64_t pred_results = 0;        // the learned model's estimates (batched method, 0 without it)
    uint64_t pred_candidates = 0;
    uint64_t* d_cost = nullptr;       // batched pre-pass: per-query work estimates
    const uint8_t* side = nullptr;    // R-S join: side byte of every record (JoinArgs.side)
    std::string ns;                   // buffer-name namespace ("" or a captured graph's own "g<id>.")
    std::string pfx(const char* name) const { return ns + "j" + std::to_string(slot) + "." + name; }
};

// Stage drivers (join.cu)
// R-S join input (rsjoin.cu): the union of R and S in memory order, the side
// of every union record (0 = R, 1 = S) and its index within that side.
struct RsInput {
    fgss_sets_view view{};               // the union, device memory
    uint8_t* side = nullptr;
    uint32_t* orig = nullptr;
    uint64_t nr = 0, ns = 0;
    const uint32_t* rid = nullptr;       // the sides' record ids on the device (or null)
    const uint32_t* sid = nullptr;
};
RsInput rs_union(Ctx& c, const fgss_sets_view& r, const fgss_sets_view& s);
// After join_output: pairs as (index in R, index in S), sorted by that.
void rs_output(Ctx& c, JoinState& J, const RsInput& u);

// Queues the input validation and the per-record counts of one join.  With
// check=false the caller synchronizes the stream once for a whole batch and
// then calls join_check_input for every join before any kernel reads tokens.
void join_setup(Ctx& c, JoinState& J, const fgss_sets_view& v, const fgss_join_opts& o, int slot, bool check = true);
// The part of join_setup both methods share: options, the input's copy to the
// device (host input), the bound tables and the JoinArgs fields that need no
// per-join buffer.
void join_setup_host(Ctx& c, JoinState& J, const fgss_sets_view& v, const fgss_join_opts& o, int slot);
void join_check_input(Ctx& c, JoinState& J);
void check_input_status(uint32_t st);  // throws on the input-validation bits
// Host copies of a join's status word and counters; throws on bad input or a
// filter-table overflow.
void apply_status(JoinState& J, uint32_t st, const unsigned long long* stats);
void join_index(Ctx& c, JoinState& J);
void join_plain_filter_verify(Ctx& c, JoinState& J, bool want_cand);
void join_features(Ctx& c, JoinState& J, float* d_feat);
void join_finish_status(Ctx& c, JoinState& J);  // D2H of status + stats, throws on bad input
void join_output(Ctx& c, JoinState& J, uint64_t* keys, uint32_t* vals, const uint64_t* d_n, uint64_t n_cap);

// Scratch of the global-memory accumulator kernel (k_probe_heavy) for `slots`
// CTAs of a join of n records, in the buffer namespace `prefix`: the always-zero
// per-source counters (zeroed when allocated) and the other per-query arrays.
struct HeavyScratch {
    uint32_t* zero = nullptr;
    uint32_t* aux = nullptr;
    uint64_t zero_words = 0, aux_words = 0;
};
HeavyScratch heavy_scratch(Ctx& c, const std::string& prefix, uint64_t n, uint32_t slots, bool capture);

// The batched method's batch: every join's per-record arrays are slices
// [roff[j], roff[j+1]) of batch-level buffers and every stage is one launch
// for the whole batch (tiles of one join per CTA, tiles.cuh).  Buffers are
// named under the context's batch namespace (c.bpfx).
struct Batch {
    std::vector<JoinState*> js;
    std::vector<uint64_t> roff;        // nj + 1: first record of each join
    uint64_t R = 0;                    // records of the batch
    uint64_t E = 0, P = 0;             // index entries, probe windows (read back by batch_prep)
    uint32_t n_max = 0;                // records of the largest join
    uint32_t terms_max = 0;
    TileMap rec{};                     // tiles of 256 records (device arrays)
    JoinArgs* d_args = nullptr;        // nj
    uint32_t* status = nullptr;        // nj x 8 (ST_* bits, longest record, heavy count, result count)
    unsigned long long* stats = nullptr;  // nj x SS_N
    uint64_t* d_e = nullptr;           // nj x 2: index entries per join
    uint32_t *icnt = nullptr, *pcnt = nullptr;  // R + 1: index / probe prefix per record
    uint32_t *ioff = nullptr, *poff = nullptr;  // R + 1: their exclusive scans (totals at R)
    uint32_t* send = nullptr;          // nj x 65537
    uint32_t* heavy_q = nullptr;       // R + 1
    // output columns (batch_filter_verify): join j's at out_off[j]
    std::vector<uint64_t> out_off;
    uint64_t out_cap = 0;
    uint32_t *oq = nullptr, *os = nullptr, *oidq = nullptr, *oids = nullptr, *oo = nullptr;
    float* osim = nullptr;
};

// Host-side decisions of one batched run, recorded eagerly and reused when the
// same batch is captured into a CUDA graph (batch.cu).
struct BatchPlan {
    bool capture = false;             // issue device work only, with these decisions
    TuneEntry te;
    uint64_t E_cap = 0, P_cap = 0;    // index entries, probe windows the buffers hold
    std::vector<uint32_t> K;          // work items per join
    uint64_t nitems = 0;
    std::vector<uint64_t> res_cap;    // result slots per join
    uint64_t cbuf_cap = 0;            // chunk-boundary words
    uint32_t heavy_slots = 0;
};
// Setup of every join (join_setup_host, with the slot each JoinState holds),
// the batch's buffers, the per-record counts and input validation of the whole
// batch (one launch each) and the index and probe totals, read back with one
// wait; throws on bad input.  Runs eagerly: a captured graph starts after it.
void batch_prep(Ctx& c, Batch& B, const std::vector<JoinState*>& js, const fgss_sets_view* views,
                const fgss_join_opts* opts);
// The inverted index of every join: one entry scatter, one sort by (join,
// term), one list pass.  E_cap: entries the buffers hold (>= B.E).
void batch_index(Ctx& c, Batch& B, uint64_t E_cap);
void batched_filter_verify(Ctx& c, Batch& B, bool use_model, BatchPlan* plan = nullptr);
// Status words and counters of every join to the host (one copy, one wait).
void batch_finish_status(Ctx& c, Batch& B);
// Per-query work estimates of a one-join batch (its index built), copied to
// host `out` (n values).
void batch_query_costs(Ctx& c, Batch& B, bool use_model, uint64_t* out);

// Autotuner (tune.cu): workload class of a join, the shapes to try, the
// cache file.
std::string tune_key(uint64_t n, uint64_t n_tokens, float t);
extern const int kFusedShapes[][3];
extern const int kNumFusedShapes;
TuneEntry filter_entry(int filter);   // the launch shape of a requested FGSS_FILTER_* strategy
int filter_of(const TuneEntry& te);   // the FGSS_FILTER_* strategy a tuned entry amounts to
TuneEntry tune_lookup(Ctx& c, const std::string& key);
void tune_load(Ctx& c);
void tune_save(Ctx& c);

// Captured batched pipelines (api.cu): dropped when shapes or the model change.
void clear_graphs(Ctx& c);

}  // namespace fgss
