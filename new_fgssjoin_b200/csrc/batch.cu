// batch.cu -- the batched method: every join of a batch in one launch per
// stage (per-record counts, index, windows, bitmaps, chunk splits, features,
// learned estimates, work-item costs, items, one persistent fused
// filter+verify launch, one global-accumulator launch, result keys, sort,
// output), presized result buffers with an exact re-run on overflow.
#include <string.h>

#include <algorithm>
#include <cmath>

#include "batch_kernels.cuh"
#include "join.h"
#include "model.h"
#include "prims.cuh"

namespace fgss {

__global__ void k_widen(const uint32_t* in, uint64_t* out);
static_assert(kFeatures == kFeat, "model feature rows");

// Warp per record: the learned model's features of one join (training rows,
// model_api.cu), the same as the batch's k_features_mj.
__global__ void k_features(JoinArgs a, float* __restrict__ feat) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < a.n; q += warps)
        features_record(a, q, feat + (uint64_t)q * kFeatures);
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
    FGSS_R(128, 11, 896)
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
                                      {128, 11, 768}, {256, 11, 768},  {256, 12, 768}, {128, 11, 896}};
extern const int kNumFusedShapes = 12;

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
    FGSS_F(128, 11, 896)
    FGSS_F(256, 11, 768)
    FGSS_F(256, 12, 768)
#undef FGSS_F
    if (sided) launch_fused<64, 9, 768, true>(c, d_args, d_fargs, items, n_items, counter, te.ctas_per_sm);
    else launch_fused<64, 9, 768, false>(c, d_args, d_fargs, items, n_items, counter, te.ctas_per_sm);
}

namespace {

constexpr uint32_t kRecTile = 256;  // records per tile of the per-record stages (thread per record in the MLP)

// Uploads the tile map of joins [off[j], off[j+1]) in tiles of `tile` to the
// device buffer `name` (through a pinned buffer of its own, so a captured
// graph's copy node always reads this map).
TileMap upload_tiles(Ctx& c, const std::string& name, const std::vector<uint64_t>& off, uint32_t tile) {
    const size_t nj = off.size() - 1;
    const size_t bytes = (nj + 1) * 12;
    char* h = (char*)c.pinned(name + ".h", bytes);
    uint64_t* ho = reinterpret_cast<uint64_t*>(h);
    uint32_t* ht = reinterpret_cast<uint32_t*>(h + (nj + 1) * 8);
    uint64_t t = 0;
    for (size_t j = 0; j < nj; j++) {
        ho[j] = off[j];
        ht[j] = (uint32_t)t;
        t += (off[j + 1] - off[j] + tile - 1) / tile;
    }
    ho[nj] = off[nj];
    if (t >= 0xffffffffull) fail(FGSS_ERR_UNSUPPORTED, "too many tiles in one batch");
    ht[nj] = (uint32_t)t;
    char* d = (char*)c.dev(name, bytes);
    FGSS_CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c.stream));
    TileMap m;
    m.roff = reinterpret_cast<const uint64_t*>(d);
    m.tile_off = reinterpret_cast<const uint32_t*>(d + (nj + 1) * 8);
    m.nj = (uint32_t)nj;
    m.tile = tile;
    m.ntiles = (uint32_t)t;
    return m;
}

// Every join's JoinArgs to the device, through the pinned buffer `name`.
void upload_args(Ctx& c, Batch& B, const std::string& name) {
    const size_t nj = B.js.size();
    JoinArgs* h = c.pinnedT<JoinArgs>(name, nj);
    for (size_t j = 0; j < nj; j++) h[j] = B.js[j]->args;
    FGSS_CK(cudaMemcpyAsync(B.d_args, h, nj * sizeof(JoinArgs), cudaMemcpyHostToDevice, c.stream));
}

unsigned tile_grid(Ctx& c, const TileMap& m, unsigned per_sm = 16) {
    return std::max<unsigned>(1, std::min<unsigned>(m.ntiles, (unsigned)c.num_sms * per_sm));
}

template <typename K>
void index_sort(Ctx& c, Batch& B, uint64_t E_cap, int tbits, int jbits, const uint64_t* d_E, const uint64_t* d_loff,
                uint32_t* list, uint2* ent) {
    const std::string& p = c.bpfx;
    K* key = c.devT<K>(p + "b.ix.key", E_cap + 1);
    uint64_t* val = c.devT<uint64_t>(p + "b.ix.val", E_cap + 1);
    k_index_entries_mj<K><<<tile_grid(c, B.rec), 256, 0, c.stream>>>(B.d_args, B.rec, B.ioff, (uint32_t)tbits, key,
                                                                      val);
    FGSS_LAUNCH_CK();
    radix_sort<K, uint64_t>(c, key, val, E_cap, d_E, 0, tbits + jbits, (p + "b.ixsort").c_str());
    k_index_lists_mj<K><<<grid_for(E_cap, 256, c.num_sms * 32), 256, 0, c.stream>>>(
        B.d_args, key, val, d_E, (uint32_t)tbits, d_loff, list, ent);
    FGSS_LAUNCH_CK();
}

// The batch's pre-pass, first part (index built): windows of every probe
// token (exact per-query work), the learned model's estimates (model) and the
// work-item cost of every query (window entries + 4 x predicted candidates +
// size) with its exclusive prefix in cpre (total at cpre[R]).  d_sums:
// [0, nj) cost totals, [nj, 2nj) predicted results, [2nj, 3nj) predicted
// candidates, [3nj] chunk-boundary words for slot tables of cap_entries.
struct Prepass {
    uint2* win = nullptr;
    uint32_t* wpre = nullptr;
    uint32_t* wtot = nullptr;
    uint4* meta = nullptr;
    uint64_t* cost = nullptr;
    uint64_t* cpre = nullptr;
    uint64_t* d_sums = nullptr;
};

Prepass batch_prepass(Ctx& c, Batch& B, uint32_t cap_entries, uint64_t P_cap, bool model) {
    const size_t nj = B.js.size();
    const std::string& p = c.bpfx;
    const uint64_t R = B.R;
    Prepass pp;
    pp.win = c.devT<uint2>(p + "b.win", P_cap + 1);
    pp.wpre = c.devT<uint32_t>(p + "b.wpre", P_cap + 1);
    pp.wtot = c.devT<uint32_t>(p + "b.wtot", R + 1);
    pp.meta = c.devT<uint4>(p + "b.meta", R + 1);
    float* feat = c.devT<float>(p + "b.feat", (R + 1) * kFeatures);
    uint32_t* pred = c.devT<uint32_t>(p + "b.pred", R + 1);
    pp.cost = c.devT<uint64_t>(p + "b.cost", R + 1);
    pp.cpre = c.devT<uint64_t>(p + "b.cpre", R + 1);
    pp.d_sums = c.devT<uint64_t>(p + "b.sums", 3 * nj + 2);
    FGSS_CK(cudaMemsetAsync(pp.d_sums, 0, (3 * nj + 2) * 8, c.stream));
    if (R == 0) return pp;
    const unsigned g = tile_grid(c, B.rec);
    k_windows_mj<<<g, 256, 0, c.stream>>>(B.d_args, B.rec, B.poff, pp.win, pp.wpre, pp.wtot, pp.meta);
    FGSS_LAUNCH_CK();
    if (model) {
        k_features_mj<<<g, 256, 0, c.stream>>>(B.d_args, B.rec, feat);
        FGSS_LAUNCH_CK();
        model_predict_tiles(c, feat, B.rec, pred, pp.d_sums + nj, pp.d_sums + 2 * nj);
    }
    k_cost_mj<<<g, 256, 0, c.stream>>>(B.d_args, B.rec, pp.wtot, model ? pred : nullptr, cap_entries, pp.cost,
                                       (unsigned long long*)(pp.d_sums + 3 * nj));
    FGSS_LAUNCH_CK();
    exclusive_scan<uint64_t>(c, pp.cost, pp.cpre, R, nullptr, pp.cpre + R, (p + "b.scan.c").c_str());
    k_join_cost_totals<<<grid_for(nj, 128), 128, 0, c.stream>>>(B.rec.roff, (uint32_t)nj, pp.cpre, pp.d_sums);
    FGSS_LAUNCH_CK();
    return pp;
}

// Second part: every record's token bitmap and the chunk splits of the
// queries whose windows exceed cap_entries, into a boundary buffer of
// cbuf_cap words (a query that finds it full is bisected by the fused kernel
// instead); returns the fused kernel's per-join arguments on the device.
FusedArgs* batch_filters(Ctx& c, Batch& B, const Prepass& pp, uint32_t cap_entries, uint64_t cbuf_cap) {
    const size_t nj = B.js.size();
    const std::string& p = c.bpfx;
    const uint64_t R = B.R;
    uint2* qchunk = c.devT<uint2>(p + "b.qchunk", R + 1);
    uint32_t* cbuf = c.devT<uint32_t>(p + "b.cbuf", cbuf_cap + 1);
    std::vector<uint64_t> boff(nj + 1, 0);
    std::vector<uint32_t> bmw(nj);
    for (size_t j = 0; j < nj; j++) {
        bmw[j] = bitmap_words(B.js[j]->in.n_tokens, B.js[j]->in.n_sets);
        boff[j + 1] = boff[j] + (uint64_t)bmw[j] * B.js[j]->in.n_sets;
    }
    uint4* bmap = c.devT<uint4>(p + "b.bmap", boff[nj] + 4);
    FusedArgs* hf = c.pinnedT<FusedArgs>(p + "b.hf", nj);
    for (size_t j = 0; j < nj; j++) {
        FusedArgs& f = hf[j];
        f.poff = B.poff + B.roff[j];
        f.win = pp.win;
        f.wpre = pp.wpre;
        f.smin = B.js[j]->lut.smin;
        f.meta = pp.meta + B.roff[j];
        f.qchunk = qchunk + B.roff[j];
        f.cbuf = cbuf;
        f.bmap = bmap + boff[j];
        f.bmw = bmw[j];
    }
    FusedArgs* d_fargs = c.devT<FusedArgs>(p + "b.fargs", nj);
    FGSS_CK(cudaMemcpyAsync(d_fargs, hf, nj * sizeof(FusedArgs), cudaMemcpyHostToDevice, c.stream));
    unsigned long long* cused = c.devT<unsigned long long>(p + "b.cused", 1);
    FGSS_CK(cudaMemsetAsync(cused, 0, 8, c.stream));
    if (R == 0) return d_fargs;
    const unsigned g = tile_grid(c, B.rec);
    k_bitmaps_mj<<<g, 256, 0, c.stream>>>(B.d_args, d_fargs, B.rec);
    FGSS_LAUNCH_CK();
    k_chunks_mj<<<g, 256, 0, c.stream>>>(B.d_args, d_fargs, B.rec, pp.wtot, cap_entries, cbuf, cbuf_cap, cused);
    FGSS_LAUNCH_CK();
    return d_fargs;
}

// The batch's launch shape: the tuned shape of its most expensive join (the
// lowest threshold, then the most records), or the one of a requested strategy.
TuneEntry batch_shape(Ctx& c, const Batch& B) {
    if (c.tune_force) return *c.tune_force;
    size_t lead = 0;
    for (size_t i = 1; i < B.js.size(); i++)
        if (B.js[i]->t < B.js[lead]->t || (B.js[i]->t == B.js[lead]->t && B.js[i]->in.n_sets > B.js[lead]->in.n_sets))
            lead = i;
    const JoinState& L = *B.js[lead];
    if (L.filter != FGSS_FILTER_AUTO) return filter_entry(L.filter);
    return tune_lookup(c, tune_key(L.in.n_sets, L.in.n_tokens, L.t));
}

}  // namespace

void batch_prep(Ctx& c, Batch& B, const std::vector<JoinState*>& js, const fgss_sets_view* views,
                const fgss_join_opts* opts) {
    const size_t nj = js.size();
    const std::string& p = c.bpfx;
    B.js = js;
    B.roff.assign(nj + 1, 0);
    B.n_max = 0;
    B.terms_max = 0;
    uint64_t T = 0;
    for (size_t j = 0; j < nj; j++) {
        JoinState& J = *js[j];
        fgss_sets_view v = views[j];
        if (!v.on_device) {
            // the same host arrays as an earlier join of the batch: copied to the device once
            for (size_t k = 0; k < j; k++) {
                const fgss_sets_view& w = views[k];
                if (!w.on_device && w.id == v.id && w.pos == v.pos && w.len == v.len && w.tokens == v.tokens &&
                    w.n_sets == v.n_sets && w.n_tokens == v.n_tokens) {
                    v = js[k]->in;
                    v.n_terms = views[j].n_terms;
                    break;
                }
            }
        }
        join_setup_host(c, J, v, opts[j], J.slot);
        B.roff[j + 1] = B.roff[j] + J.in.n_sets;
        B.n_max = std::max<uint32_t>(B.n_max, (uint32_t)J.in.n_sets);
        B.terms_max = std::max<uint32_t>(B.terms_max, J.in.n_terms);
        T += J.in.n_tokens;
    }
    B.R = B.roff[nj];
    // per-record offsets are 32-bit: the caller splits larger batches
    if (T >= 0xffffffffull || B.R >= 0xffffffffull) fail(FGSS_ERR_UNSUPPORTED, "a batch of 2^32 or more tokens");
    B.status = c.devT<uint32_t>(p + "b.status", nj * 8);
    B.stats = c.devT<unsigned long long>(p + "b.stats", nj * SS_N);
    B.d_e = c.devT<uint64_t>(p + "b.E", nj * 2);
    B.icnt = c.devT<uint32_t>(p + "b.icnt", B.R + 1);
    B.pcnt = c.devT<uint32_t>(p + "b.pcnt", B.R + 1);
    B.ioff = c.devT<uint32_t>(p + "b.ioff", B.R + 1);
    B.poff = c.devT<uint32_t>(p + "b.poff", B.R + 1);
    B.send = c.devT<uint32_t>(p + "b.send", nj * 65537);
    B.heavy_q = c.devT<uint32_t>(p + "b.heavy_q", B.R + 1);
    B.d_args = c.devT<JoinArgs>(p + "b.args", nj);
    FGSS_CK(cudaMemsetAsync(B.status, 0, nj * 32, c.stream));
    FGSS_CK(cudaMemsetAsync(B.stats, 0, nj * SS_N * 8, c.stream));
    for (size_t j = 0; j < nj; j++) {
        JoinState& J = *js[j];
        J.status = B.status + 8 * j;
        J.stats = B.stats + SS_N * j;
        J.maxlen = J.status + 1;
        J.d_e = B.d_e + 2 * j;
        J.icnt = B.icnt + B.roff[j];
        J.pcnt = B.pcnt + B.roff[j];
        JoinArgs& a = J.args;
        a.status = J.status;
        a.stats = J.stats;
        a.send = B.send + 65537ull * j;
        a.heavy_q = B.heavy_q + B.roff[j];
        a.heavy_count = J.status + 2;
        a.res_count = J.status + 3;
    }
    B.rec = upload_tiles(c, p + "b.rec", B.roff, kRecTile);
    upload_args(c, B, p + "b.ha0");
    if (B.R) {
        k_prep_mj<<<tile_grid(c, B.rec), 256, 0, c.stream>>>(B.d_args, B.rec, B.icnt, B.pcnt);
        FGSS_LAUNCH_CK();
        k_send_mj<<<grid_for((uint64_t)nj << 16, 256, c.num_sms * 32), 256, 0, c.stream>>>(B.d_args, (uint32_t)nj,
                                                                                          B.send);
        FGSS_LAUNCH_CK();
        exclusive_scan<uint32_t>(c, B.icnt, B.ioff, B.R, nullptr, B.ioff + B.R, (p + "b.scan.i").c_str());
        exclusive_scan<uint32_t>(c, B.pcnt, B.poff, B.R, nullptr, B.poff + B.R, (p + "b.scan.p").c_str());
    } else {
        FGSS_CK(cudaMemsetAsync(B.ioff, 0, 4, c.stream));
        FGSS_CK(cudaMemsetAsync(B.poff, 0, 4, c.stream));
    }
    // one wait for the whole batch: no kernel reads tokens through caller
    // offsets before they are validated
    uint32_t* h = c.pinnedT<uint32_t>(p + "b.hprep", nj * 8 + 2);
    FGSS_CK(cudaMemcpyAsync(h, B.status, nj * 32, cudaMemcpyDeviceToHost, c.stream));
    FGSS_CK(cudaMemcpyAsync(h + nj * 8, B.ioff + B.R, 4, cudaMemcpyDeviceToHost, c.stream));
    FGSS_CK(cudaMemcpyAsync(h + nj * 8 + 1, B.poff + B.R, 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    for (size_t j = 0; j < nj; j++)
        if (js[j]->in.n_sets) check_input_status(h[8 * j]);
    B.E = h[nj * 8];
    B.P = h[nj * 8 + 1];
}

void batch_index(Ctx& c, Batch& B, uint64_t E_cap) {
    const size_t nj = B.js.size();
    const std::string& p = c.bpfx;
    if (E_cap < B.E) fail(FGSS_ERR_CUDA, "index buffers below the batch's entry count");
    const int tbits = bits_for((uint64_t)B.terms_max + 1);
    const int jbits = bits_for(nj);
    // join j's list offsets: n_terms + 1 entries from loff[j], positions in
    // the batch's entry arrays
    uint64_t* hl = c.pinnedT<uint64_t>(p + "b.hloff", nj + 1);
    hl[0] = 0;
    for (size_t j = 0; j < nj; j++) hl[j + 1] = hl[j] + B.js[j]->in.n_terms + 1;
    const uint64_t L = hl[nj];
    uint64_t* d_loff = c.devT<uint64_t>(p + "b.loff", nj + 1);
    FGSS_CK(cudaMemcpyAsync(d_loff, hl, (nj + 1) * 8, cudaMemcpyHostToDevice, c.stream));
    uint32_t* list = c.devT<uint32_t>(p + "b.list", L + 1);
    uint2* ent = c.devT<uint2>(p + "b.ent", E_cap + 1);
    for (size_t j = 0; j < nj; j++) {
        JoinArgs& a = B.js[j]->args;
        a.list_off = list + hl[j];
        a.ent = ent;
    }
    // a join without entries keeps these zero offsets (empty lists)
    FGSS_CK(cudaMemsetAsync(list, 0, L * 4, c.stream));
    FGSS_CK(cudaMemsetAsync(B.d_e, 0, nj * 16, c.stream));
    if (B.R) {
        uint64_t* d_E = c.devT<uint64_t>(p + "b.dE", 2);
        k_widen<<<1, 1, 0, c.stream>>>(B.ioff + B.R, d_E);
        FGSS_LAUNCH_CK();
        k_join_entries<<<grid_for(nj, 128), 128, 0, c.stream>>>(B.rec.roff, (uint32_t)nj, B.ioff, B.d_e);
        FGSS_LAUNCH_CK();
        if (tbits + jbits <= 32) index_sort<uint32_t>(c, B, E_cap, tbits, jbits, d_E, d_loff, list, ent);
        else index_sort<uint64_t>(c, B, E_cap, tbits, jbits, d_E, d_loff, list, ent);
    }
    upload_args(c, B, p + "b.ha1");
}

void batch_query_costs(Ctx& c, Batch& B, bool use_model, uint64_t* out) {
    if (B.R == 0) return;
    const TuneEntry te = batch_shape(c, B);
    const Prepass pp = batch_prepass(c, B, (1u << te.hash_log2) / 4 * 3, B.P, use_model && c.model);
    FGSS_CK(cudaMemcpyAsync(out, pp.cost, B.R * 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
}

// Runs the fused filter+verify over every join of the batch (index built).
//
// With a plan in record mode the host-side decisions of this run (launch
// shape, buffer sizes, work items per join, result capacities, heavy-path
// slots) are kept; in capture mode (plan->capture) the same device work is
// issued with those decisions and without any host synchronization, so the
// stream can be captured into a CUDA graph and replayed on later calls.
void batched_filter_verify(Ctx& c, Batch& B, bool use_model, BatchPlan* plan) {
    const size_t nj = B.js.size();
    std::vector<JoinState*>& joins = B.js;
    const bool capture = plan && plan->capture;
    const std::string& p = c.bpfx;
    const TuneEntry te = capture ? plan->te : batch_shape(c, B);
    const uint32_t cap_entries = (1u << te.hash_log2) / 4 * 3;  // chunk capacity of the chosen kernel shape
    const uint64_t P_cap = plan ? plan->P_cap : B.P;
    if (P_cap < B.P) fail(FGSS_ERR_CUDA, "window buffers below the batch's probe-token count");
    const bool model = use_model && c.model;
    const Prepass pp = batch_prepass(c, B, cap_entries, P_cap, model);

    // work items: ~256 per resident CTA over the whole batch (a few queries per
    // item at 100k records), split by cost share and handed out longest first,
    // so the dynamic queue ends with short items
    std::vector<uint32_t> K(nj, 0);
    uint64_t nitems = 0;
    uint64_t* hsum = c.pinnedT<uint64_t>(p + "b.hsum", 3 * nj + 2);
    if (capture) {
        K = plan->K;
        nitems = plan->nitems;
    } else {
        FGSS_CK(cudaMemcpyAsync(hsum, pp.d_sums, (3 * nj + 2) * 8, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        for (size_t i = 0; i < nj; i++) {
            if (!model || joins[i]->res_cap_hint) continue;
            joins[i]->pred_results = hsum[nj + i];
            joins[i]->pred_candidates = hsum[2 * nj + i];
        }
        uint64_t grand = 0;
        for (size_t i = 0; i < nj; i++) grand += hsum[i];
        const uint64_t want = (uint64_t)256 * fused_resident_ctas(c, te);
        for (size_t i = 0; i < nj; i++) {
            const uint64_t n = joins[i]->in.n_sets;
            if (n == 0) continue;
            uint64_t k = grand ? (want * hsum[i] + grand - 1) / grand : 1;
            k = std::max<uint64_t>(1, std::min<uint64_t>(k, n));
            K[i] = (uint32_t)k;
            nitems += k;
        }
    }
    if (nitems >= 0xffffffffull) fail(FGSS_ERR_UNSUPPORTED, "too many work items");
    // chunk boundaries: exactly the words the splits take (the plan's size in
    // a capture; a replay on other data that needs more bisects instead)
    const uint64_t cbuf_cap = capture ? plan->cbuf_cap : std::min<uint64_t>(hsum[3 * nj], 0xfffffff0ull);
    if (plan && !capture) plan->cbuf_cap = cbuf_cap;
    FusedArgs* d_fargs = batch_filters(c, B, pp, cap_entries, cbuf_cap);
    uint32_t* hk = c.pinnedT<uint32_t>(p + "b.hkoff", nj + 1);
    hk[0] = 0;
    for (size_t i = 0; i < nj; i++) hk[i + 1] = hk[i] + K[i];
    uint32_t* d_koff = c.devT<uint32_t>(p + "b.koff", nj + 1);
    FGSS_CK(cudaMemcpyAsync(d_koff, hk, (nj + 1) * 4, cudaMemcpyHostToDevice, c.stream));
    uint4* items = c.devT<uint4>(p + "b.items", nitems + 1);
    if (nitems) {
        uint32_t* ikey = c.devT<uint32_t>(p + "b.ikey", nitems + 1);
        uint32_t* ival = c.devT<uint32_t>(p + "b.ival", nitems + 1);
        k_items_mj<<<grid_for(nitems, 128), 128, 0, c.stream>>>(B.rec.roff, d_koff, (uint32_t)nj, (uint32_t)nitems,
                                                                 pp.cpre, pp.d_sums, items, ikey, ival);
        FGSS_LAUNCH_CK();
        if (nitems > 1) {
            // longest-processing-time order: sort items by descending cost
            uint4* sorted = c.devT<uint4>(p + "b.items2", nitems + 1);
            radix_sort<uint32_t, uint32_t>(c, ikey, ival, nitems, nullptr, 0, 16, (p + "b.isort").c_str());
            k_permute_items<<<grid_for(nitems, 128), 128, 0, c.stream>>>(items, ival, nitems, sorted);
            FGSS_LAUNCH_CK();
            items = sorted;
        }
    }

    bool sided = false;
    for (size_t i = 0; i < nj; i++) sided |= joins[i]->args.side != nullptr;
    uint32_t* counter = c.devT<uint32_t>(p + "b.counter", 4 + nj);
    uint32_t* hst = c.pinnedT<uint32_t>(p + "b.hst", nj * 8);
    std::vector<uint64_t> cap(nj, 0);
    uint32_t slots = 0;
    // (inside a capture the events must be external record nodes to be timed at replay)
    const unsigned rec_flags = capture ? cudaEventRecordExternal : 0u;
    for (int attempt = 0;; attempt++) {
        // result buffers: the caller's size, the learned estimate (x1.5 +
        // slack), the last size seen for this slot, or the exact count after
        // an overflow
        std::vector<uint64_t> capoff(nj + 1, 0);
        for (size_t i = 0; i < nj; i++) {
            JoinState& J = *joins[i];
            if (capture) {
                cap[i] = plan->res_cap[i];
            } else {
                auto itc = c.tune.find(J.pfx("rescap"));
                const uint64_t last = itc != c.tune.end() ? (uint64_t)itc->second.ctas_per_sm : 0;
                uint64_t v;
                if (J.res_cap_hint) v = J.res_cap_hint;
                else if (J.res_cap_user) v = J.res_cap_user;
                else if (model) v = std::max<uint64_t>((uint64_t)((double)hsum[nj + i] * 1.5) + 4096, last);
                else v = std::max<uint64_t>(J.in.n_sets + 4096, last);
                cap[i] = std::min<uint64_t>(v, 0xfffffff0ull);
            }
            capoff[i + 1] = capoff[i] + cap[i];
        }
        uint32_t* res_q = c.devT<uint32_t>(p + "b.res.q", capoff[nj] + 1);
        uint32_t* res_s = c.devT<uint32_t>(p + "b.res.s", capoff[nj] + 1);
        uint32_t* res_o = c.devT<uint32_t>(p + "b.res.o", capoff[nj] + 1);
        for (size_t i = 0; i < nj; i++) {
            JoinArgs& a = joins[i]->args;
            a.res_cap = (uint32_t)cap[i];
            a.heavy_min_qp = te.heavy_min_probe > 0 ? (uint32_t)te.heavy_min_probe : 0xffffffffu;
            a.res_q = res_q + capoff[i];
            a.res_s = res_s + capoff[i];
            a.res_o = res_o + capoff[i];
        }
        upload_args(c, B, p + "b.ha2");
        FGSS_CK(cudaMemsetAsync(counter, 0, (4 + nj) * 4, c.stream));
        FGSS_CK(cudaEventRecordWithFlags(c.ev[4], c.stream, rec_flags));
        if (nitems) fused_launch(c, te, B.d_args, d_fargs, items, (uint32_t)nitems, counter, sided);
        FGSS_CK(cudaEventRecordWithFlags(c.ev[5], c.stream, rec_flags));
        c.probe_timed = true;
        // queries deferred to the global-memory accumulator: one persistent
        // launch for every join.  Eagerly only when some were queued; under a
        // plan always, with scratch for a fixed slot count (a launch whose
        // queues are empty returns at once).
        uint32_t max_nh = 0;
        if (!capture) {
            FGSS_CK(cudaMemcpyAsync(hst, B.status, nj * 32, cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            for (size_t i = 0; i < nj; i++) max_nh = std::max(max_nh, hst[8 * i + 2]);
        }
        const uint32_t all_slots = std::min<uint32_t>(std::max<uint32_t>(B.n_max, 1), (uint32_t)c.num_sms);
        slots = capture ? plan->heavy_slots : plan ? all_slots : std::min<uint32_t>(max_nh, (uint32_t)c.num_sms);
        if (slots) {
            const HeavyScratch hs = heavy_scratch(c, p, B.n_max, slots, capture);
            FGSS_CK(cudaEventRecordWithFlags(c.ev[6], c.stream, rec_flags));
            k_probe_heavy<MODE_FUSED, 512><<<slots, 512, 0, c.stream>>>(B.d_args, 0, (uint32_t)nj, hs.zero,
                                                                        hs.zero_words, hs.aux, hs.aux_words,
                                                                        counter + 4);
            FGSS_LAUNCH_CK();
            FGSS_CK(cudaEventRecordWithFlags(c.ev[7], c.stream, rec_flags));
            c.heavy_timed = true;
        }
        if (capture) break;
        FGSS_CK(cudaMemcpyAsync(hst, B.status, nj * 32, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        bool over = false;
        for (size_t i = 0; i < nj; i++) {
            JoinState& J = *joins[i];
            const uint32_t got = hst[8 * i + 3];
            if (got > cap[i]) {
                // The learned (or remembered) capacity was too small: the kernel
                // kept counting, so the batch re-runs with the exact size.  A
                // plan keeps that exact size for the captured batch.
                J.res_cap_hint = got;
                J.overflow_retries++;
                over = true;
            }
        }
        if (!over) break;
        if (attempt) fail(FGSS_ERR_CUDA, "result buffers overflowed at their exact size");
        k_clear_filter_state_mj<<<(unsigned)std::min<size_t>(nj, 1024), 32, 0, c.stream>>>(B.d_args, (uint32_t)nj);
        FGSS_LAUNCH_CK();
    }
    if (plan && !capture) {
        plan->te = te;
        plan->K = K;
        plan->nitems = nitems;
        plan->heavy_slots = slots;
        plan->res_cap = cap;
    }

    // results: join j's in the output columns from out_off[j] (its result
    // count eagerly, its capacity under a plan, so a captured graph finds
    // every buffer at the size it has now)
    std::vector<uint64_t> rcap(nj);
    for (size_t i = 0; i < nj; i++) {
        JoinState& J = *joins[i];
        if (capture) {
            rcap[i] = cap[i];
            continue;
        }
        const uint32_t got = hst[8 * i + 3];
        J.n_res = got;
        J.res_cap_hint = 0;
        // remember a sufficient capacity for the next call on this slot
        c.tune[J.pfx("rescap")].ctas_per_sm = (int)std::min<uint64_t>((uint64_t)got + got / 4 + 1024, 0x7fffffff);
        rcap[i] = plan ? cap[i] : got;
    }
    B.out_off.assign(nj + 1, 0);
    for (size_t i = 0; i < nj; i++) B.out_off[i + 1] = B.out_off[i] + rcap[i];
    B.out_cap = B.out_off[nj];
    const uint64_t oc = B.out_cap;
    B.oq = c.devT<uint32_t>(p + "b.o.q", oc + 1);
    B.os = c.devT<uint32_t>(p + "b.o.s", oc + 1);
    B.oidq = c.devT<uint32_t>(p + "b.o.idq", oc + 1);
    B.oids = c.devT<uint32_t>(p + "b.o.ids", oc + 1);
    B.oo = c.devT<uint32_t>(p + "b.o.o", oc + 1);
    B.osim = c.devT<float>(p + "b.o.sim", oc + 1);
    for (size_t i = 0; i < nj; i++) {
        JoinState& J = *joins[i];
        const uint64_t o = B.out_off[i];
        J.oq = B.oq + o;
        J.os = B.os + o;
        J.oidq = B.oidq + o;
        J.oids = B.oids + o;
        J.oo = B.oo + o;
        J.osim = B.osim + o;
    }
    if (oc == 0) return;
    const TileMap rt = upload_tiles(c, p + "b.rt", B.out_off, 256);
    uint64_t* resoff = c.devT<uint64_t>(p + "b.resoff", nj + 2);
    uint64_t* d_n = resoff + nj + 1;
    k_result_offsets<<<1, 1024, 0, c.stream>>>(B.d_args, (uint32_t)nj, resoff, d_n);
    FGSS_LAUNCH_CK();
    // sort keys join << 2qb | q << qb | s: only the bits that vary
    const int qb = bits_for(B.n_max), jb = bits_for(nj);
    if (2 * qb + jb > 64) fail(FGSS_ERR_UNSUPPORTED, "result keys of more than 64 bits");
    uint64_t* key = c.devT<uint64_t>(p + "b.rkey", oc + 1);
    uint32_t* val = c.devT<uint32_t>(p + "b.rval", oc + 1);
    k_result_keys_mj<<<tile_grid(c, rt), 256, 0, c.stream>>>(B.d_args, rt, resoff, (uint32_t)qb, key, val);
    FGSS_LAUNCH_CK();
    radix_sort<uint64_t, uint32_t>(c, key, val, oc, d_n, 0, 2 * qb + jb, (p + "b.rsort").c_str());
    k_result_out_mj<<<grid_for(oc, 256, c.num_sms * 32), 256, 0, c.stream>>>(
        B.d_args, key, val, d_n, resoff, rt.roff, (uint32_t)qb, B.oq, B.os, B.oidq, B.oids, B.oo, B.osim);
    FGSS_LAUNCH_CK();
}

void batch_finish_status(Ctx& c, Batch& B) {
    const size_t nj = B.js.size();
    uint32_t* h = c.pinnedT<uint32_t>(c.bpfx + "b.hfin", nj * 8);
    unsigned long long* hs = c.pinnedT<unsigned long long>(c.bpfx + "b.hfin.stats", nj * SS_N);
    uint64_t* he = c.pinnedT<uint64_t>(c.bpfx + "b.hfin.E", nj * 2);
    FGSS_CK(cudaMemcpyAsync(h, B.status, nj * 32, cudaMemcpyDeviceToHost, c.stream));
    FGSS_CK(cudaMemcpyAsync(hs, B.stats, nj * SS_N * 8, cudaMemcpyDeviceToHost, c.stream));
    FGSS_CK(cudaMemcpyAsync(he, B.d_e, nj * 16, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    for (size_t j = 0; j < nj; j++) {
        B.js[j]->n_entries = he[2 * j];
        B.js[j]->n_res = h[8 * j + 3];
        apply_status(*B.js[j], h[8 * j], hs + SS_N * j);
    }
}

}  // namespace fgss
