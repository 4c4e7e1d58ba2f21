// batch.cu -- the batched method: per-query features and cost, balanced work
// items, one persistent fused filter+verify launch over every join of a
// batch, presized result buffers with an exact re-run on overflow.
#include <string.h>

#include <algorithm>
#include <cmath>

#include "fused_kernels.cuh"
#include "join.h"
#include "model.h"
#include "prims.cuh"

namespace fgss {

// Per query: features of the cost model and the heuristic cost
// (sum of the probe tokens' full list lengths, plus the query size).
__global__ void k_features(JoinArgs a, float t, float* __restrict__ feat, uint32_t* __restrict__ cost) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    for (uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < a.n; q += warps) {
        uint32_t lq = a.len[q];
        uint32_t qp = lq <= 65535u ? a.probe[lq] : 0;
        const uint32_t* qt = a.tok + a.pos[q];
        unsigned long long sum = 0;
        uint32_t mx = 0;
        float slog = 0.f;
        for (uint32_t j = lane; j < qp; j += 32) {
            uint32_t w = __ldg(qt + j);
            uint32_t l = __ldg(a.list_off + w + 1) - __ldg(a.list_off + w);
            sum += l;
            mx = max(mx, l);
            slog += log1pf((float)l);
        }
        sum = warp_sum(sum);
        mx = __reduce_max_sync(kFull, mx);
        slog = warp_sum(slog);
        if (lane == 0) {
            uint32_t send = lq <= 65535u ? a.send[lq] : q + 1;
            uint32_t win = send > q + 1 ? send - q - 1 : 0;
            float* f = feat + (uint64_t)q * kFeat;
            f[0] = log1pf((float)lq);
            f[1] = log1pf((float)qp);
            f[2] = log1pf((float)sum);
            f[3] = log1pf((float)mx);
            f[4] = qp ? slog / (float)qp : 0.f;
            f[5] = log1pf((float)win);
            f[6] = a.n ? (float)q / (float)a.n : 0.f;
            f[7] = t;
            unsigned long long c = sum + lq;
            cost[q] = (uint32_t)min(c, 0x3fffffffull);
        }
    }
}

// Work items of one join: item k = queries with exclusive cost prefix in
// [k*target, (k+1)*target).
__global__ void k_items(const uint64_t* __restrict__ pre, uint32_t n, const uint64_t* __restrict__ d_total, uint32_t K,
                        uint32_t join, uint4* __restrict__ items) {
    const uint64_t total = *d_total;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        uint64_t target = (total + K - 1) / K;
        auto first_ge = [&](uint64_t x) {
            uint32_t lo = 0, hi = n;
            while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                if (pre[mid] < x) lo = mid + 1;
                else hi = mid;
            }
            return lo;
        };
        uint32_t b = k == 0 ? 0 : first_ge(k * target);
        uint32_t e = k + 1 == K ? n : first_ge((k + 1) * target);
        items[k] = make_uint4(join, b, max(b, e), 0);
    }
}

// Item sort keys: ~cost (so ascending order = descending cost), value = item index.
// Sort key of a work item: its cost as a float's exponent and top 7 mantissa
// bits (the longest-first order needs no more), complemented so an ascending
// sort puts the costliest first; 16 bits, two radix passes.
__global__ void k_item_keys(const uint64_t* __restrict__ pre, uint32_t n, const uint64_t* __restrict__ d_total,
                            const uint4* __restrict__ items, uint32_t K, uint32_t base, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ val) {
    const uint64_t total = *d_total;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        const uint4 it = items[k];
        const uint64_t b = it.y < n ? pre[it.y] : total;
        const uint64_t e = it.z < n ? pre[it.z] : total;
        key[base + k] = (~__float_as_uint((float)(e - b)) >> 16) & 0xffffu;
        val[base + k] = base + k;
    }
}

__global__ void k_permute_items(const uint4* __restrict__ items, const uint32_t* __restrict__ order, uint64_t n,
                                uint4* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = items[order[i]];
}

template <int NT, int HLOG, int RT>
static int resident_ctas(Ctx& c) {
    int occ = 0;
    FGSS_CK(cudaFuncSetAttribute(k_fused<NT, HLOG, RT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)FusedLayout<HLOG>::bytes));
    FGSS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fused<NT, HLOG, RT, false>, NT,
                                                          FusedLayout<HLOG>::bytes));
    return std::max(occ, 1) * c.num_sms;
}

int fused_resident_ctas(Ctx& c, const TuneEntry& te) {
#define FGSS_R(NT, HL, RT) \
    if (te.threads == NT && te.hash_log2 == HL && te.regs_rt == RT) return resident_ctas<NT, HL, RT>(c);
    FGSS_R(32, 8, 1024)
    FGSS_R(32, 9, 1024)
    FGSS_R(64, 9, 1024)
    FGSS_R(64, 9, 768)
    FGSS_R(64, 10, 1024)
    FGSS_R(128, 9, 1024)
    FGSS_R(128, 10, 1024)
    FGSS_R(128, 10, 768)
    FGSS_R(128, 11, 768)
    FGSS_R(256, 11, 768)
    FGSS_R(256, 12, 768)
#undef FGSS_R
    return resident_ctas<64, 9, 768>(c);
}

template <int NT, int HLOG, int RT, bool SIDED>
static void launch_fused(Ctx& c, const JoinArgs* d_args, const FusedArgs* d_fargs, const uint4* items,
                         uint32_t n_items, uint32_t* counter, int ctas_per_sm) {
    static bool attr = false;
    const size_t smem = FusedLayout<HLOG>::bytes;
    if (!attr) {
        FGSS_CK(cudaFuncSetAttribute(k_fused<NT, HLOG, RT, SIDED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        attr = true;
    }
    int occ = 0;
    FGSS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fused<NT, HLOG, RT, SIDED>, NT, smem));
    if (occ < 1) occ = 1;
    const int per = ctas_per_sm > 0 ? std::min(occ, ctas_per_sm) : occ;
    const unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)per * c.num_sms, std::max<uint32_t>(n_items, 1));
    k_fused<NT, HLOG, RT, SIDED><<<grid, NT, smem, c.stream>>>(d_args, d_fargs, items, n_items, counter);
    FGSS_LAUNCH_CK();
}

// Launch shapes the autotuner chooses from: CTA size, slot-table log2 size,
// resident threads per SM the register budget is sized for.
extern const int kFusedShapes[][3] = {{32, 8, 1024},  {32, 9, 1024},  {64, 9, 1024},   {64, 9, 768},
                                      {64, 10, 1024}, {128, 9, 1024}, {128, 10, 1024}, {128, 10, 768},
                                      {128, 11, 768}, {256, 11, 768},  {256, 12, 768}};
extern const int kNumFusedShapes = 11;

// The launch shape that stands for a requested filter strategy.
TuneEntry filter_entry(int filter) {
    TuneEntry te;
    te.threads = filter == FGSS_FILTER_WARP ? 32 : 128;
    te.hash_log2 = filter == FGSS_FILTER_WARP ? 9 : 11;
    te.regs_rt = filter == FGSS_FILTER_WARP ? 1024 : 768;
    te.ctas_per_sm = 0;
    te.heavy_min_probe = filter == FGSS_FILTER_GLOBAL ? 1 : 0;
    return te;
}

// The strategy a tuned entry amounts to.
int filter_of(const TuneEntry& te) {
    return te.heavy_min_probe == 1 ? FGSS_FILTER_GLOBAL : te.threads == 32 ? FGSS_FILTER_WARP : FGSS_FILTER_CTA;
}

// sided: the batch is an R-S join (its records carry a side byte)
void fused_launch(Ctx& c, const TuneEntry& te, const JoinArgs* d_args, const FusedArgs* d_fargs, const uint4* items,
                  uint32_t n_items, uint32_t* counter, bool sided) {
#define FGSS_F(NT, HL, RT)                                                                               \
    if (te.threads == NT && te.hash_log2 == HL && te.regs_rt == RT) {                                    \
        if (sided) launch_fused<NT, HL, RT, true>(c, d_args, d_fargs, items, n_items, counter, te.ctas_per_sm); \
        else launch_fused<NT, HL, RT, false>(c, d_args, d_fargs, items, n_items, counter, te.ctas_per_sm);      \
        return;                                                                                          \
    }
    FGSS_F(32, 8, 1024)
    FGSS_F(32, 9, 1024)
    FGSS_F(64, 9, 1024)
    FGSS_F(64, 9, 768)
    FGSS_F(64, 10, 1024)
    FGSS_F(128, 9, 1024)
    FGSS_F(128, 10, 1024)
    FGSS_F(128, 10, 768)
    FGSS_F(128, 11, 768)
    FGSS_F(256, 11, 768)
    FGSS_F(256, 12, 768)
#undef FGSS_F
    if (sided) launch_fused<64, 9, 768, true>(c, d_args, d_fargs, items, n_items, counter, te.ctas_per_sm);
    else launch_fused<64, 9, 768, false>(c, d_args, d_fargs, items, n_items, counter, te.ctas_per_sm);
}

// Work-item cost of a query: exact window entries + a verification estimate.
__global__ void k_cost(const uint32_t* __restrict__ wtot, const uint32_t* __restrict__ len,
                       const uint32_t* __restrict__ pred_cand, uint32_t n, uint32_t q_lo, uint32_t q_hi,
                       uint64_t* __restrict__ cost) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        if (q < q_lo || q >= q_hi) {  // outside this shard: no work
            cost[q] = 0;
            continue;
        }
        unsigned long long v = (unsigned long long)wtot[q] + len[q];
        if (pred_cand) v += 4ull * pred_cand[q];
        cost[q] = v;
    }
}

// Resets the filter's counters and overflow bit of one join before a re-run
// (the input-validation bits and the probe-token count stay).
__global__ void k_clear_filter_state(uint32_t* status, unsigned long long* stats) {
    if (threadIdx.x == 0) {
        status[0] &= ~(uint32_t)(ST_RES_OVERFLOW | ST_HEAVY_OVERFLOW | ST_HASH_FULL);
        status[2] = 0;
        status[3] = 0;
    }
    if (threadIdx.x < SS_N && threadIdx.x != SS_PROBE) stats[threadIdx.x] = 0;
}

// The batched method's pre-pass of one join (index built already): windows of
// every probe token (exact per-query work), bitmaps, chunk splits for slot
// tables of cap_entries, the learned model's estimates (use_model), and the
// work-item cost of every query (window entries + 4 x predicted candidates +
// size) with its exclusive prefix in `pre` and total in d_total.
FusedArgs join_prepass(Ctx& c, JoinState& J, uint32_t cap_entries, bool use_model, uint64_t* d_pred_res,
                       uint64_t* d_pred_cand, uint64_t* pre, uint64_t* d_total) {
    const uint64_t n = J.in.n_sets;
    float* feat = c.devT<float>(J.pfx("feat"), (n + 1) * kFeat);
    uint64_t* cost = c.devT<uint64_t>(J.pfx("cost"), n + 1);
    uint32_t* fcost = c.devT<uint32_t>(J.pfx("fcost"), n + 1);
    uint32_t* poff = c.devT<uint32_t>(J.pfx("poff"), n + 1);
    uint2* win = c.devT<uint2>(J.pfx("win"), J.in.n_tokens + 1);
    uint32_t* wpre = c.devT<uint32_t>(J.pfx("wpre"), J.in.n_tokens + 1);
    uint32_t* wtot = c.devT<uint32_t>(J.pfx("wtot"), n + 1);
    uint32_t* pred = c.devT<uint32_t>(J.pfx("pred"), n + 1);
    uint4* meta = c.devT<uint4>(J.pfx("meta"), n + 1);
    const uint32_t bmw = bitmap_words(J.in.n_tokens, n);
    uint4* bmap = c.devT<uint4>(J.pfx("bmap"), (uint64_t)bmw * n + 4);
    uint2* qchunk = c.devT<uint2>(J.pfx("qchunk"), n + 1);
    const uint64_t cbuf_cap = 2 * J.in.n_tokens + (1u << 20);  // overflowing queries bisect instead
    uint32_t* cbuf = c.devT<uint32_t>(J.pfx("cbuf"), cbuf_cap);
    FusedArgs f;
    f.poff = poff;
    f.win = win;
    f.wpre = wpre;
    f.smin = J.lut.smin;
    f.meta = meta;
    f.qchunk = qchunk;
    f.cbuf = cbuf;
    f.bmap = bmap;
    f.bmw = bmw;
    J.d_cost = cost;
    if (n == 0) return f;
    // windows of every probe token (exact per-query work), chunk splits, then
    // features and the learned estimate, then the work-item cost prefix
    exclusive_scan<uint32_t>(c, J.pcnt, poff, n, nullptr, (uint32_t*)nullptr, J.pfx("scan.p").c_str());
    unsigned long long* cused = reinterpret_cast<unsigned long long*>(J.status + 4);
    FGSS_CK(cudaMemsetAsync(cused, 0, 8, c.stream));
    k_windows<<<grid_for(n * 32, 256, c.num_sms * 64), 256, 0, c.stream>>>(J.args, poff, win, wpre, wtot, meta);
    FGSS_LAUNCH_CK();
    k_bitmaps<<<grid_for(n * 32, 256, c.num_sms * 64), 256, 0, c.stream>>>(J.args, bmap, bmw);
    FGSS_LAUNCH_CK();
    k_chunks<<<grid_for(n * 32, 256, c.num_sms * 64), 256, 0, c.stream>>>(J.args, poff, win, wtot, cap_entries, qchunk,
                                                                        cbuf, cbuf_cap, cused);
    FGSS_LAUNCH_CK();
    const bool model = use_model && c.model && !J.res_cap_hint;
    if (model) {
        k_features<<<grid_for(n * 32, 256, c.num_sms * 32), 256, 0, c.stream>>>(J.args, J.t, feat, fcost);
        FGSS_LAUNCH_CK();
        model_predict(c, feat, n, pred, d_pred_res, d_pred_cand);
    }
    k_cost<<<grid_for(n, 256, c.num_sms * 8), 256, 0, c.stream>>>(wtot, J.in.len, model ? pred : nullptr, (uint32_t)n,
                                                                   J.args.q_lo, J.args.q_hi, cost);
    FGSS_LAUNCH_CK();
    exclusive_scan<uint64_t>(c, cost, pre, n, nullptr, d_total, J.pfx("scan.cost").c_str());
    return f;
}

// Per-query work estimates of one join (index built already), to host `out`:
// the costs the batched method balances its work items by.
void join_query_costs(Ctx& c, JoinState& J, bool use_model, uint64_t* out) {
    const uint64_t n = J.in.n_sets;
    if (n == 0) return;
    const TuneEntry te = tune_lookup(c, tune_key(n, J.in.n_tokens, J.t));
    uint64_t* d_tot = c.devT<uint64_t>(J.pfx("qc.tot"), 4);
    FGSS_CK(cudaMemsetAsync(d_tot, 0, 32, c.stream));
    uint64_t* pre = c.devT<uint64_t>(J.pfx("cpre"), n + 1);
    join_prepass(c, J, (1u << te.hash_log2) / 2, use_model, d_tot + 1, d_tot + 2, pre, d_tot);
    FGSS_CK(cudaMemcpyAsync(out, J.d_cost, n * 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
}

// Runs the fused filter+verify over every join (their index built already).
//
// With a plan in record mode the host-side decisions of this run (launch
// shape, work items per join, result capacities, heavy-path slots, grid) are
// kept; in capture mode (plan->capture) the same device work is issued with
// those decisions and without any host synchronization, so the stream can be
// captured into a CUDA graph and replayed on later calls.
void batched_filter_verify(Ctx& c, std::vector<JoinState*>& joins, bool use_model, BatchPlan* plan) {
    const size_t nj = joins.size();
    const bool capture = plan && plan->capture;
    // d_tot: [0, nj) cost totals, [nj, 2nj) predicted results, [2nj, 3nj) predicted candidates
    uint64_t* d_tot = c.devT<uint64_t>(c.bpfx + "b.tot", nj * 3 + 2);
    std::vector<uint64_t*> pre(nj);
    FGSS_CK(cudaMemsetAsync(d_tot, 0, (nj * 3 + 2) * 8, c.stream));
    FusedArgs* hf = c.pinnedT<FusedArgs>(c.bpfx + "b.hf", nj);
    TuneEntry te;
    if (capture) {
        te = plan->te;
    } else {
        // one launch shape for the batch: the tuned shape of its most expensive
        // join (the lowest threshold, then the most records)
        size_t lead = 0;
        for (size_t i = 1; i < nj; i++)
            if (joins[i]->t < joins[lead]->t ||
                (joins[i]->t == joins[lead]->t && joins[i]->in.n_sets > joins[lead]->in.n_sets))
                lead = i;
        te = c.tune_force ? *c.tune_force
                          : tune_lookup(c, tune_key(joins[lead]->in.n_sets, joins[lead]->in.n_tokens, joins[lead]->t));
        if (!c.tune_force && joins[lead]->filter != FGSS_FILTER_AUTO) te = filter_entry(joins[lead]->filter);
    }
    const uint32_t cap_entries = (1u << te.hash_log2) / 2;  // chunk capacity of the chosen kernel shape
    for (size_t i = 0; i < nj; i++) {
        JoinState& J = *joins[i];
        pre[i] = c.devT<uint64_t>(J.pfx("cpre"), J.in.n_sets + 1);
        hf[i] = join_prepass(c, J, cap_entries, use_model, &d_tot[nj + i], &d_tot[2 * nj + i], pre[i], &d_tot[i]);
    }
    FusedArgs* d_fargs = c.devT<FusedArgs>(c.bpfx + "b.fargs", nj);
    FGSS_CK(cudaMemcpyAsync(d_fargs, hf, nj * sizeof(FusedArgs), cudaMemcpyHostToDevice, c.stream));
    std::vector<uint32_t> K(nj, 0);
    uint64_t nitems = 0;
    std::vector<uint64_t> htot(3 * nj + 2, 0);
    if (capture) {
        K = plan->K;
        nitems = plan->nitems;
    } else {
        FGSS_CK(cudaMemcpyAsync(htot.data(), d_tot, (3 * nj + 2) * 8, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        for (size_t i = 0; i < nj; i++) {
            if (!(use_model && c.model && !joins[i]->res_cap_hint)) continue;
            joins[i]->pred_results = htot[nj + i];
            joins[i]->pred_candidates = htot[2 * nj + i];
        }
        uint64_t grand = 0;
        for (size_t i = 0; i < nj; i++) grand += htot[i];
        // ~256 items per resident CTA over the whole batch (a few queries per item at
        // 100k records), split by cost share and handed out longest first, so the
        // dynamic queue ends with short items
        const uint64_t want = (uint64_t)256 * fused_resident_ctas(c, te);
        for (size_t i = 0; i < nj; i++) {
            const uint64_t n = joins[i]->in.n_sets;
            if (n == 0) continue;
            uint64_t k = grand ? (want * htot[i] + grand - 1) / grand : 1;
            k = std::max<uint64_t>(1, std::min<uint64_t>(k, n));
            K[i] = (uint32_t)k;
            nitems += k;
        }
    }
    uint4* items = c.devT<uint4>(c.bpfx + "b.items", nitems + 1);
    uint64_t off = 0;
    for (size_t i = 0; i < nj; i++) {
        if (!K[i]) continue;
        JoinState& J = *joins[i];
        k_items<<<grid_for(K[i], 128), 128, 0, c.stream>>>(pre[i], (uint32_t)J.in.n_sets, &d_tot[i], K[i],
                                                            (uint32_t)i, items + off);
        FGSS_LAUNCH_CK();
        off += K[i];
    }
    if (nitems > 1) {
        // longest-processing-time order: sort items by descending cost
        uint32_t* ikey = c.devT<uint32_t>(c.bpfx + "b.ikey", nitems + 1);
        uint32_t* ival = c.devT<uint32_t>(c.bpfx + "b.ival", nitems + 1);
        uint4* sorted = c.devT<uint4>(c.bpfx + "b.items2", nitems + 1);
        uint64_t off2 = 0;
        for (size_t i = 0; i < nj; i++) {
            if (!K[i]) continue;
            k_item_keys<<<grid_for(K[i], 128), 128, 0, c.stream>>>(pre[i], (uint32_t)joins[i]->in.n_sets, &d_tot[i],
                                                                    items + off2, K[i], (uint32_t)off2, ikey, ival);
            FGSS_LAUNCH_CK();
            off2 += K[i];
        }
        radix_sort<uint32_t, uint32_t>(c, ikey, ival, nitems, nullptr, 0, 16, (c.bpfx + "b.isort").c_str());
        k_permute_items<<<grid_for(nitems, 128), 128, 0, c.stream>>>(items, ival, nitems, sorted);
        FGSS_LAUNCH_CK();
        items = sorted;
    }
    // result buffers: the caller's size, the learned estimate (x1.5 + slack),
    // or the last size seen for this slot
    JoinArgs* d_args = c.devT<JoinArgs>(c.bpfx + "b.args", nj);
    JoinArgs* hargs = c.pinnedT<JoinArgs>(c.bpfx + "b.hargs", nj);
    for (size_t i = 0; i < nj; i++) {
        JoinState& J = *joins[i];
        const uint64_t n = J.in.n_sets;
        uint64_t cap;
        if (capture) {
            cap = plan->res_cap[i];
        } else {
            auto itc = c.tune.find(J.pfx("rescap"));
            const uint64_t last = itc != c.tune.end() ? (uint64_t)itc->second.ctas_per_sm : 0;
            if (J.res_cap_hint) {
                cap = J.res_cap_hint;
            } else if (J.res_cap_user) {
                cap = J.res_cap_user;
            } else if (use_model && c.model) {
                // predicted results x 1.5 + slack, or the size this slot needed last time if larger
                cap = std::max<uint64_t>((uint64_t)((double)htot[nj + i] * 1.5) + 4096, last);
            } else {
                cap = std::max<uint64_t>(n + 4096, last);
            }
            cap = std::min<uint64_t>(cap, 0xfffffff0ull);
        }
        JoinArgs& a = J.args;
        a.res_cap = (uint32_t)cap;
        a.heavy_min_qp = te.heavy_min_probe > 0 ? (uint32_t)te.heavy_min_probe : 0xffffffffu;
        a.res_q = c.devT<uint32_t>(J.pfx("res.q"), cap + 1);
        a.res_s = c.devT<uint32_t>(J.pfx("res.s"), cap + 1);
        a.res_o = c.devT<uint32_t>(J.pfx("res.o"), cap + 1);
        a.res_count = J.status + 3;
        FGSS_CK(cudaMemsetAsync(a.heavy_count, 0, 8, c.stream));  // heavy_count + res_count
        hargs[i] = a;
    }
    FGSS_CK(cudaMemcpyAsync(d_args, hargs, nj * sizeof(JoinArgs), cudaMemcpyHostToDevice, c.stream));
    uint32_t* counter = c.devT<uint32_t>(c.bpfx + "b.counter", 4 + nj);
    FGSS_CK(cudaMemsetAsync(counter, 0, (4 + nj) * 4, c.stream));
    // (inside a capture the events must be external record nodes to be timed at replay)
    const unsigned rec_flags = capture ? cudaEventRecordExternal : 0u;
    FGSS_CK(cudaEventRecordWithFlags(c.ev[4], c.stream, rec_flags));
    bool sided = false;
    for (size_t i = 0; i < nj; i++) sided |= joins[i]->args.side != nullptr;
    if (nitems) fused_launch(c, te, d_args, d_fargs, items, (uint32_t)nitems, counter, sided);
    FGSS_CK(cudaEventRecordWithFlags(c.ev[5], c.stream, rec_flags));
    c.probe_timed = true;
    // heavy queries: one persistent launch per join.  Eagerly only when some
    // were queued; under a plan always, with scratch for a fixed slot count
    // (a launch with an empty queue returns at once).
    uint32_t* hbuf = c.pinnedT<uint32_t>(c.bpfx + "b.hq", 2 * nj + 2);
    if (!capture) {
        for (size_t i = 0; i < nj; i++)
            FGSS_CK(cudaMemcpyAsync(hbuf + 2 * i, joins[i]->status + 2, 8, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    }
    for (size_t i = 0; i < nj; i++) {
        JoinState& J = *joins[i];
        uint32_t slots;
        if (capture) {
            slots = plan->heavy_slots[i];
        } else {
            const uint32_t nh = hbuf[2 * i];
            slots = plan ? std::min<uint32_t>((uint32_t)std::max<uint64_t>(J.in.n_sets, 1), (uint32_t)c.num_sms)
                         : std::min<uint32_t>(nh, (uint32_t)c.num_sms);
            if (!nh && !plan) slots = 0;
        }
        if (!slots) continue;
        const HeavyScratch hs = heavy_scratch(c, c.bpfx, J.in.n_sets, slots, capture);
        k_probe_heavy<MODE_FUSED, 512><<<slots, 512, 0, c.stream>>>(d_args, (uint32_t)i, hs.zero, hs.zero_words, hs.aux,
                                                                    hs.aux_words, counter + 4 + i);
        FGSS_LAUNCH_CK();
    }
    if (plan && !capture) {
        plan->te = te;
        plan->K = K;
        plan->nitems = nitems;
        plan->heavy_slots.assign(nj, 0);
        for (size_t i = 0; i < nj; i++)
            plan->heavy_slots[i] =
                std::min<uint32_t>((uint32_t)std::max<uint64_t>(joins[i]->in.n_sets, 1), (uint32_t)c.num_sms);
        plan->res_cap.assign(nj, 0);
    }
    if (capture) {
        // results sorted at full capacity; the host reads the counts after replay
        for (size_t i = 0; i < nj; i++) {
            JoinState& J = *joins[i];
            uint64_t* keys = c.devT<uint64_t>(J.pfx("rkey"), (uint64_t)J.args.res_cap + 1);
            uint32_t* vals = c.devT<uint32_t>(J.pfx("rval"), (uint64_t)J.args.res_cap + 1);
            J.d_nres = c.devT<uint64_t>(J.pfx("nres"), 2);
            k_result_keys<<<grid_for(J.args.res_cap, 256, c.num_sms * 32), 256, 0, c.stream>>>(
                J.args.res_q, J.args.res_s, J.args.res_o, J.status + 3, J.args.res_cap, keys, vals, J.d_nres);
            FGSS_LAUNCH_CK();
            join_output(c, J, keys, vals, J.d_nres, J.args.res_cap);
        }
        return;
    }
    // results: overflow -> exact re-run of that join with the exact capacity
    for (size_t i = 0; i < nj; i++)
        FGSS_CK(cudaMemcpyAsync(hbuf + 2 * i, joins[i]->status + 3, 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    const std::vector<uint32_t> gots = [&] {
        std::vector<uint32_t> g(nj);
        for (size_t i = 0; i < nj; i++) g[i] = hbuf[2 * i];
        return g;
    }();
    for (size_t i = 0; i < nj; i++) {
        JoinState& J = *joins[i];
        const uint32_t got = gots[i];
        if (got > J.args.res_cap) {
            // The learned (or remembered) capacity was too small: the kernel kept
            // counting, so re-run this join alone with the exact size.  A plan
            // keeps that exact size for the captured batch.
            J.res_cap_hint = got;
            J.overflow_retries++;
            k_clear_filter_state<<<1, 32, 0, c.stream>>>(J.status, J.stats);
            FGSS_LAUNCH_CK();
            std::vector<JoinState*> one{&J};
            batched_filter_verify(c, one, false, nullptr);
            if (plan) plan->res_cap[i] = J.args.res_cap;
            continue;
        }
        if (plan) plan->res_cap[i] = J.args.res_cap;
        // remember a sufficient capacity for the next call on this slot
        J.res_cap_hint = 0;
        c.tune[J.pfx("rescap")].ctas_per_sm = (int)std::min<uint64_t>((uint64_t)got + got / 4 + 1024, 0x7fffffff);
        uint64_t* keys = c.devT<uint64_t>(J.pfx("rkey"), (uint64_t)J.args.res_cap + 1);
        uint32_t* vals = c.devT<uint32_t>(J.pfx("rval"), (uint64_t)J.args.res_cap + 1);
        J.d_nres = c.devT<uint64_t>(J.pfx("nres"), 2);
        if (got) {
            k_result_keys<<<grid_for(got, 256, c.num_sms * 32), 256, 0, c.stream>>>(
                J.args.res_q, J.args.res_s, J.args.res_o, J.status + 3, J.args.res_cap, keys, vals, J.d_nres);
            FGSS_LAUNCH_CK();
        } else {
            FGSS_CK(cudaMemsetAsync(J.d_nres, 0, 8, c.stream));
        }
        // under a plan, the output stage is sized at capacity so the captured
        // graph finds every buffer at the size it has now
        join_output(c, J, keys, vals, J.d_nres, plan ? (uint64_t)J.args.res_cap : (uint64_t)got);
        J.n_res = got;
    }
}

}  // namespace fgss
