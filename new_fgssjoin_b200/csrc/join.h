// join.h -- host driver of the self-join (plain and batched methods).
#pragma once

#include <vector>

#include "bounds.h"
#include "ctx.h"
#include "join_kernels.cuh"

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
    uint64_t res_cap_hint = 0;   // exact result count after an overflow
    uint64_t res_cap_user = 0;   // caller's result capacity (fgss_join_opts.result_capacity)
    uint32_t overflow_retries = 0;
    uint32_t status_host = 0;
    unsigned long long stats_host[SS_N] = {};
    std::vector<uint32_t> cand_host;  // (q, s, partial) triples when requested
    uint64_t pred_results = 0;        // the learned model's estimates (batched method, 0 without it)
    uint64_t pred_candidates = 0;
    uint64_t* d_cost = nullptr;       // batched pre-pass: per-query work estimates
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
void join_check_input(Ctx& c, JoinState& J);
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

// Host-side decisions of one batched run, recorded eagerly and reused when the
// same batch is captured into a CUDA graph (batch.cu).
struct BatchPlan {
    bool capture = false;             // issue device work only, with these decisions
    TuneEntry te;
    std::vector<uint32_t> K;          // work items per join
    uint64_t nitems = 0;
    std::vector<uint64_t> res_cap;    // result slots per join
    std::vector<uint32_t> heavy_slots;
};
void batched_filter_verify(Ctx& c, std::vector<JoinState*>& joins, bool use_model, BatchPlan* plan = nullptr);
// Per-query work estimates of one join (its index built), copied to host `out` (n values).
void join_query_costs(Ctx& c, JoinState& J, bool use_model, uint64_t* out);

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
