// join_kernels.cuh -- device side of the self-join: prefix lengths, inverted
// index, candidate filtering, verification and result compaction.
//
// Reference path (RafaelQuirino/new_fgssjoin), per stage:
//   prefix lengths     src/fgssjoin/data.cu:241-257  (select_midpref_tokens_kernel)
//   inverted index     src/fgssjoin/index.cu:276-342 (midpref/df_count/inverted_index kernels)
//   filtering          src/fgssjoin/filtering.cu:76-141 (thread per query, dense short
//                      score matrix, size + positional filter) and compaction.cu:8-17
//   verification       src/fgssjoin/checking.cu:93-175 (thread per candidate merge)
//   compaction/output  src/fgssjoin/checking.cu:556-595, block.cu:184-197
//
// B200 design.  No block x block score matrix: a CTA owns one query at a time
// and accumulates its candidates in a shared-memory hash table (a
// global-memory dense accumulator for the few queries too large for it).
// Sources are limited to an id window [q+1, send) found by binary search in
// each inverted list (lists are sorted by source id, sources by descending
// size), so entries outside the size filter are never read.  Each hash slot
// keeps (source, matches, last match position): the number of prefix matches
// is the reference's partial score, the last match reproduces its positional
// filter exactly (the bound it tests at every match is non-increasing, so it
// fails at some match iff it fails at the last) and lets verification resume
// right after it.  Verification is warp-cooperative: 32 source tokens per
// step, each lane binary-searches the query's tokens (staged in shared memory
// by the fused kernel) and the warp counts matches with ballot + popc.
#pragma once

#include "common.cuh"

namespace fgss {

constexpr uint32_t kEmpty = 0xffffffffu;

// status bits (per join)
enum : uint32_t {
    ST_UNSORTED = 1u << 0,   // record sizes not non-increasing in memory order
    ST_SKIP_ALL = 1u << 1,   // unsorted input whose one-tile skip test prunes everything
    ST_TOO_LONG = 1u << 2,   // a record longer than 65535 tokens
    ST_BAD_TOKENS = 1u << 3, // tokens not strictly ascending inside a record / >= n_terms
    ST_RES_OVERFLOW = 1u << 4,
    ST_HEAVY_OVERFLOW = 1u << 5,
    ST_HASH_FULL = 1u << 6,
    ST_BAD_OFFSETS = 1u << 7, // a record's pos + len runs past n_tokens
};

// stats slots (per join, unsigned long long)
enum {
    SS_CANDIDATES = 0,
    SS_INTERSECTIONS,
    SS_RESULTS,
    SS_WINDOW,
    SS_VERIFIED,
    SS_HEAVY,
    SS_PROBE,
    SS_MERGED,
    SS_QTOK,   // tokens of the query records the fused kernel staged
    SS_N
};

struct JoinArgs {
    const uint32_t* pos;
    const uint32_t* len;
    const uint32_t* tok;
    uint32_t n;
    uint32_t n_terms;
    uint64_t n_tokens;
    uint32_t* status;          // ST_* bits
    unsigned long long* stats; // SS_* counters
    // bound tables (bounds.h)
    const uint16_t* probe;
    const uint16_t* index;
    const uint32_t* minsz;
    const uint32_t* maxsz;
    const uint32_t* cand_min;
    const uint32_t* inter_min;
    const uint32_t* need;
    const uint32_t* send;      // per query length: end of the source id window (sorted input)
    const uint32_t* lmin;      // per query length: smallest source size the size filter keeps
    const uint32_t* id;        // record ids (null: the memory index)
    float thr;                 // the join's threshold
    // inverted index
    const uint32_t* list_off;  // [n_terms + 1]
    const uint2* ent;          // per entry: (source record, source size << 16 | position of the token
                               // in the source); sources ascending within a list
    // plain method
    uint32_t* vcnt;            // count pass: per query, candidates that need a merge
    uint32_t* ccnt;            // count pass: per query, candidates (reference definition)
    uint32_t* wcnt;            // count pass: per query, window entries read
    const uint32_t* voff;      // fill pass: exclusive scan of vcnt
    uint4* cand;               // fill pass: (q, s, matches, last_q << 16 | last_s)
    // fused method
    uint32_t* res_q;
    uint32_t* res_s;
    uint32_t* res_o;
    uint32_t res_cap;
    uint32_t* res_count;
    // queries deferred to the global-memory accumulator
    uint32_t* heavy_q;
    uint32_t* heavy_count;
    uint32_t heavy_cap;
    uint32_t join_id;
    uint32_t q_lo;             // queries processed: [q_lo, q_hi) (a shard of the join)
    uint32_t q_hi;
    uint32_t heavy_min_qp;     // fused method: probe prefixes this long go to the global accumulator
    // R-S join: one byte per record (0 = R, 1 = S); pairs within one side are
    // skipped before any filter.  nullptr for a self-join.
    const uint8_t* side;
};

// ------------------------------------------------------------ small helpers

// first index in [lo, hi) with a[i] >= x (a ascending)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint32_t x) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// first entry in [lo, hi) whose source is >= x (sources ascending)
__device__ __forceinline__ uint32_t lower_bound_src(const uint2* __restrict__ e, uint32_t lo, uint32_t hi, uint32_t x) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&e[mid].x) < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// first index in [lo, hi) of smem/generic array with a[i] > x
__device__ __forceinline__ uint32_t upper_bound_gen(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t x) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool contains_gen(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t x) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t v = a[mid];
        if (v == x) return true;
        if (v < x) lo = mid + 1;
        else hi = mid;
    }
    return false;
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t s, int hlog) { return (s * 0x9E3779B1u) >> (32 - hlog); }

// Size filter of filtering.cu:111-120 for one (query, source) pair.
__device__ __forceinline__ bool size_ok(const JoinArgs& a, uint32_t lq, uint32_t ls) {
    return !(ls < a.minsz[lq] || ls > a.maxsz[lq] || lq < a.minsz[ls] || lq > a.maxsz[ls]);
}

// Warp-cooperative overlap of q[qa:lq) and s[sa:ls) added to `base`; stops
// as soon as base + matches + (what is left) < need.  q may be shared or
// global memory.  All 32 lanes must call it; returns the same value on all.
__device__ __forceinline__ uint32_t warp_merge_count(const uint32_t* q, uint32_t qa, uint32_t lq,
                                                     const uint32_t* __restrict__ s, uint32_t sa, uint32_t ls,
                                                     uint32_t base, uint32_t need) {
    const uint32_t lane = lane_id();
    uint32_t cnt = base;
    for (uint32_t b = sa; b < ls && qa < lq; b += 32) {
        uint32_t k = b + lane;
        bool has = k < ls;
        uint32_t x = has ? __ldg(s + k) : 0xffffffffu;
        bool found = has && contains_gen(q, qa, lq, x);
        cnt += __popc(__ballot_sync(kFull, found));
        // q tokens <= the chunk's last source token are consumed
        uint32_t last = __shfl_sync(kFull, x, (ls - b >= 32) ? 31 : (ls - b - 1));
        uint32_t nqa = 0;
        if (lane == 0) nqa = upper_bound_gen(q, qa, lq, last);
        qa = __shfl_sync(kFull, nqa, 0);
        uint32_t rs = ls > b + 32 ? ls - b - 32 : 0;
        uint32_t rq = lq - qa;
        if (cnt + min(rs, rq) < need) break;
    }
    return cnt;
}

// ------------------------------------------------------------- prefix stage

// Per record: prefix lengths (data.cu:241-257), validation of the input
// (sizes, order, tokens).  icnt / pcnt are the record's own slots.
__device__ __forceinline__ void prep_record(const JoinArgs& a, uint32_t i, uint32_t* icnt, uint32_t* pcnt,
                                            uint32_t& local_max, uint32_t& bad, unsigned long long& probe,
                                            int check_tokens) {
    const uint32_t l = a.len[i];
    local_max = max(local_max, l);
    if ((uint64_t)a.pos[i] + l > a.n_tokens) {
        bad |= ST_BAD_OFFSETS;
        *icnt = 0;
        *pcnt = 0;
        return;
    }
    if (l > 65535u) {
        bad |= ST_TOO_LONG;
        *icnt = 0;
        *pcnt = 0;
        return;
    }
    if (i + 1 < a.n && a.len[i + 1] > l) bad |= ST_UNSORTED;
    *icnt = a.index[l];
    *pcnt = a.probe[l];
    probe += a.probe[l];
    if (check_tokens) {
        const uint32_t* t = a.tok + a.pos[i];
        uint32_t prev = 0;
        for (uint32_t j = 0; j < l; j++) {
            const uint32_t v = t[j];
            if (v >= a.n_terms || (j > 0 && v <= prev)) bad |= ST_BAD_TOKENS;
            prev = v;
        }
    }
}

// Warp-collective: the warp's maximum size, status bits and probe-token count to the join.
__device__ __forceinline__ void prep_flush(const JoinArgs& a, uint32_t* maxlen, uint32_t local_max, uint32_t bad,
                                           unsigned long long probe) {
    local_max = __reduce_max_sync(kFull, local_max);
    bad = __reduce_or_sync(kFull, bad);
    probe = warp_sum(probe);
    if (lane_id() == 0) {
        if (local_max) atomicMax(maxlen, local_max);
        if (bad) atomicOr(a.status, bad);
        if (probe) atomicAdd(&a.stats[SS_PROBE], probe);
    }
}

// The one-tile skip test of block.cu:121-130 (only reachable for unsorted input).
__device__ __forceinline__ void prep_skip_test(const JoinArgs& a) {
    if (a.n == 0) return;
    const uint32_t l0 = a.len[0], ln = a.len[a.n - 1];
    if (l0 <= 65535u && ln > a.maxsz[l0]) atomicOr(a.status, ST_SKIP_ALL);
}

static __global__ void k_prep(JoinArgs a, uint32_t* __restrict__ icnt, uint32_t* __restrict__ pcnt, uint32_t* maxlen,
                              int check_tokens) {
    uint32_t local_max = 0, bad = 0;
    unsigned long long probe = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
        prep_record(a, i, icnt + i, pcnt + i, local_max, bad, probe, check_tokens);
    prep_flush(a, maxlen, local_max, bad, probe);
    if (blockIdx.x == 0 && threadIdx.x == 0) prep_skip_test(a);
}

// send[L] for every query length L: the number of records of size >= lmin[L]
// (records have non-increasing sizes).
__device__ __forceinline__ uint32_t send_of(const uint32_t* __restrict__ len, uint32_t n, uint32_t target) {
    uint32_t lo = 0, hi = n;  // first i with len[i] < target
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (len[mid] >= target) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static __global__ void k_send(const uint32_t* __restrict__ len, uint32_t n, const uint32_t* __restrict__ lmin,
                              uint32_t* __restrict__ send, uint32_t nl) {
    for (uint32_t L = blockIdx.x * blockDim.x + threadIdx.x; L < nl; L += gridDim.x * blockDim.x)
        send[L] = send_of(len, n, lmin[L]);
}

// -------------------------------------------------------------- index stage

// Index entries of one record's index prefix (warp-collective), written from
// position o: key = tag | term, value = record << 32 | size << 16 | position.
template <typename K>
__device__ __forceinline__ void index_entries_record(const JoinArgs& a, uint32_t i, uint64_t o, K tag,
                                                     K* __restrict__ key, uint64_t* __restrict__ val) {
    const uint32_t l = a.len[i];
    if (l > 65535u) return;
    const uint32_t ip = a.index[l];
    const uint32_t* t = a.tok + a.pos[i];
    for (uint32_t j = lane_id(); j < ip; j += 32) {
        key[o + j] = tag | (K)t[j];
        val[o + j] = ((uint64_t)i << 32) | (l << 16) | j;
    }
}

static __global__ void k_index_entries(JoinArgs a, const uint32_t* __restrict__ ioff, uint32_t* __restrict__ key,
                                       uint64_t* __restrict__ val) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.n; i += warps)
        index_entries_record<uint32_t>(a, i, ioff[i], 0u, key, val);
}

// After the stable sort by term: list offsets (no atomics: the thread at each
// term boundary fills the offsets of the terms it spans) and the 8-byte entries.
static __global__ void k_index_lists(const uint32_t* __restrict__ key, const uint64_t* __restrict__ val,
                              const uint64_t* __restrict__ d_e, uint32_t n_terms, uint32_t* __restrict__ list_off,
                              uint2* __restrict__ ent) {
    const uint32_t E = (uint32_t)*d_e;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (E == 0) {
        for (uint32_t w = tid; w <= n_terms; w += stride) list_off[w] = 0;
        return;
    }
    for (uint32_t k = tid; k < E; k += stride) {
        uint64_t v = val[k];
        ent[k] = make_uint2((uint32_t)(v >> 32), (uint32_t)v);
        uint32_t w = key[k];
        if (k == 0)
            for (uint32_t x = 0; x <= w; x++) list_off[x] = 0;
        uint32_t nxt = (k + 1 < E) ? key[k + 1] : n_terms;
        for (uint32_t x = w + 1; x <= nxt; x++) list_off[x] = k + 1;
    }
}

}  // namespace fgss

namespace fgss {

// ------------------------------------------------------- filter + verify

enum { MODE_COUNT = 0, MODE_FILL = 1, MODE_FUSED = 2 };

constexpr uint32_t kPCap = 1024;     // probe tokens whose windows fit in shared memory
constexpr uint32_t kQCap = 2048;     // query tokens staged in shared memory
constexpr uint32_t kBmWords = 2048;  // query term bitmap: 65536 bits
constexpr unsigned long long kEmptySlot = 0xffffffff00000000ull;

// Shared-memory layout of the light-query kernel.
//   slots u64[H]   (source << 32 | matches << 16 | last query position)
//   wlo/whi u32[kPCap]   full id window of each probe token's list
//   clo u32[kPCap], wpre u32[kPCap + 4]   the current chunk: first entry, exclusive scan of sizes
//   qtok u32[kQCap]   query tokens;  bitmap u32[kBmWords] (fused only)
template <int MODE, int HLOG>
struct ProbeLayout {
    static constexpr uint32_t H = 1u << HLOG;
    static constexpr uint32_t cap = H / 2;  // window entries per chunk (slot load <= 1/2)
    static constexpr size_t off_wlo = 8ull * H;
    static constexpr size_t off_whi = off_wlo + 4ull * kPCap;
    static constexpr size_t off_clo = off_whi + 4ull * kPCap;
    static constexpr size_t off_wpre = off_clo + 4ull * kPCap;
    static constexpr size_t off_qtok = off_wpre + 4ull * (kPCap + 4);
    static constexpr size_t off_bm = off_qtok + 4ull * kQCap;
    static constexpr size_t bytes = off_bm + (MODE == MODE_FUSED ? 4ull * kBmWords : 0);
};

struct CtaCounters {
    unsigned long long cand, inter, res, window, verified, heavy, merged;
};

__device__ __forceinline__ void flush_counters(const JoinArgs& a, const CtaCounters& c) {
    if (c.cand) atomicAdd(&a.stats[SS_CANDIDATES], c.cand);
    if (c.inter) atomicAdd(&a.stats[SS_INTERSECTIONS], c.inter);
    if (c.res) atomicAdd(&a.stats[SS_RESULTS], c.res);
    if (c.window) atomicAdd(&a.stats[SS_WINDOW], c.window);
    if (c.verified) atomicAdd(&a.stats[SS_VERIFIED], c.verified);
    if (c.heavy) atomicAdd(&a.stats[SS_HEAVY], c.heavy);
    if (c.merged) atomicAdd(&a.stats[SS_MERGED], c.merged);
}

// All lanes of a warp: sum the per-thread counters, one lane adds them.
__device__ __forceinline__ void flush_counters_warp(const JoinArgs& a, CtaCounters c) {
    c.cand = warp_sum(c.cand);
    c.inter = warp_sum(c.inter);
    c.res = warp_sum(c.res);
    c.window = warp_sum(c.window);
    c.verified = warp_sum(c.verified);
    c.heavy = warp_sum(c.heavy);
    c.merged = warp_sum(c.merged);
    if (lane_id() == 0) flush_counters(a, c);
}

// Emits one verified pair (called by one lane).
__device__ __forceinline__ void emit_result(const JoinArgs& a, uint32_t q, uint32_t s, uint32_t o) {
    uint32_t idx = atomicAdd(a.res_count, 1u);
    if (idx < a.res_cap) {
        a.res_q[idx] = q;
        a.res_s[idx] = s;
        a.res_o[idx] = o;
    } else {
        atomicOr(a.status, ST_RES_OVERFLOW);
    }
}

__device__ __forceinline__ void defer_heavy(const JoinArgs& a, uint32_t q) {
    uint32_t i = atomicAdd(a.heavy_count, 1u);
    if (i < a.heavy_cap) a.heavy_q[i] = q;
    else atomicOr(a.status, ST_HEAVY_OVERFLOW);
}

// One match (source s, query position j) into the slot table: a single 64-bit
// CAS inserts the key or bumps (matches, last position).  False if full.
__device__ __forceinline__ bool slot_add(unsigned long long* slots, uint32_t mask, int hl, uint32_t s, uint32_t j) {
    uint32_t h = hash_slot(s, hl);
    for (uint32_t it = 0; it <= mask; it++) {
        unsigned long long old = *(volatile unsigned long long*)&slots[h];
        for (;;) {
            const uint32_t key = (uint32_t)(old >> 32);
            unsigned long long nw;
            if (key == s) {
                const uint32_t lo = (uint32_t)old;
                nw = ((unsigned long long)s << 32) | ((((lo >> 16) + 1u) << 16) | max(lo & 0xffffu, j));
            } else if (key == kEmpty) {
                nw = ((unsigned long long)s << 32) | ((1u << 16) | j);
            } else {
                break;
            }
            const unsigned long long prev = atomicCAS(&slots[h], old, nw);
            if (prev == old) return true;
            old = prev;
        }
        h = (h + 1) & mask;
    }
    return false;
}

// Is the source's matching position (of query token xq) <= tau?  The position
// lies in [c - 1, ips - 1] (c matches at or before it, all in the index
// prefix); one token read decides the rest.
__device__ __forceinline__ bool smax_le(const uint32_t* __restrict__ st, int tau, uint32_t c, uint32_t ips,
                                        uint32_t xq) {
    if (tau < (int)c - 1) return false;
    if (tau >= (int)ips - 1) return true;
    return __ldg(st + tau) >= xq;
}

// Position of xq in the source's index prefix (warp-wide; xq is present).
__device__ __forceinline__ uint32_t warp_find(const uint32_t* __restrict__ st, uint32_t ips, uint32_t xq) {
    for (uint32_t b = 0; b < ips; b += 32) {
        uint32_t k = b + lane_id();
        uint32_t x = k < ips ? __ldg(st + k) : 0xffffffffu;
        uint32_t m = __ballot_sync(kFull, x == xq);
        if (m) return b + __ffs(m) - 1;
    }
    return ips;  // unreachable for a consistent index
}

// Reference-candidate and needs-merge tests of one slot (filtering.cu:125-135
// at the last match; checking.cu:110,156 bound).
struct SlotVerdict {
    bool cand, ver;
};
__device__ __forceinline__ SlotVerdict slot_verdict(const JoinArgs& a, uint32_t lq, uint32_t c, uint32_t jm, uint32_t s,
                                                    uint32_t xq) {
    const uint32_t ls = a.len[s], S = lq + ls, A = lq - jm;
    const uint32_t cm = a.cand_min[S], im = a.inter_min[S];
    const uint32_t ips = a.index[ls];
    const uint32_t* st = a.tok + a.pos[s];
    SlotVerdict v;
    v.cand = (c + A >= cm) && smax_le(st, (int)ls + (int)c - (int)cm, c, ips, xq);
    v.ver = (c + A - 1 >= im) && smax_le(st, (int)ls + (int)c - 1 - (int)im, c, ips, xq);
    return v;
}

// Thread-serial merge of a source's tokens from position p0 against the
// query's term bitmap, counting only tokens above xq (the query token of the
// last prefix match: everything at or below it was counted by the filter).
// Stops as soon as c + matches + what can still match < im.
__device__ __forceinline__ uint32_t thread_merge(const uint32_t* __restrict__ st, uint32_t p0, uint32_t ls,
                                                 uint32_t xq, uint32_t c, uint32_t qrest, uint32_t im,
                                                 const uint32_t* bm, bool exact, const uint32_t* qtok, uint32_t qa,
                                                 uint32_t lq, uint32_t* nread) {
    uint32_t cnt = c;
    uint32_t k = p0;
    auto visit = [&](uint32_t x) {
        if (x <= xq) return;
        const uint32_t b = exact ? x : ((x * 0x9E3779B1u) >> 16);
        bool hit = (bm[b >> 5] >> (b & 31)) & 1u;
        if (hit && !exact) hit = contains_gen(qtok, qa, lq, x);
        cnt += hit;
    };
    auto alive = [&](uint32_t kk) { return cnt + min(ls - kk, qrest - (cnt - c)) >= im; };
    bool go = true;
    while (k < ls && (reinterpret_cast<uintptr_t>(st + k) & 15u)) {
        if (!alive(k)) { go = false; break; }
        visit(__ldg(st + k));
        k++;
    }
    while (go && k + 4 <= ls) {
        if (!alive(k)) { go = false; break; }
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(st + k));
        visit(v.x);
        visit(v.y);
        visit(v.z);
        visit(v.w);
        k += 4;
    }
    while (go && k < ls) {
        if (!alive(k)) break;
        visit(__ldg(st + k));
        k++;
    }
    *nread = k - p0;
    return cnt;
}

// Light query on one CTA: shared-memory slot table; the id window is split
// into chunks of at most `cap` entries (depth-first bisection).  Queries
// beyond the shared-memory caps go to the heavy queue.
template <int MODE, int NT, int HLOG>
__device__ void probe_query_smem(const JoinArgs& a, uint32_t q, unsigned char* smem, CtaCounters& ctr) {
    using Lay = ProbeLayout<MODE, HLOG>;
    unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* wlo = reinterpret_cast<uint32_t*>(smem + Lay::off_wlo);
    uint32_t* whi = reinterpret_cast<uint32_t*>(smem + Lay::off_whi);
    uint32_t* clo = reinterpret_cast<uint32_t*>(smem + Lay::off_clo);
    uint32_t* wpre = reinterpret_cast<uint32_t*>(smem + Lay::off_wpre);
    uint32_t* qtok = reinterpret_cast<uint32_t*>(smem + Lay::off_qtok);
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + Lay::off_bm);
    __shared__ uint32_t s_L, s_vc, s_cand, s_sp, s_win;
    __shared__ uint32_t s_sa[48], s_sb[48];
    __shared__ uint32_t wsum[33];

    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint32_t st_bits = *a.status;
    if (st_bits & ST_SKIP_ALL) return;
    if (q < a.q_lo || q >= a.q_hi) return;
    const uint32_t lq = a.len[q];
    if (lq == 0 || lq > 65535u) return;
    const uint32_t qp = a.probe[lq];
    if (qp == 0) return;
    if (qp > kPCap || lq > kQCap) {
        if (tid == 0) defer_heavy(a, q);
        return;
    }
    const bool unsorted = (st_bits & ST_UNSORTED) != 0;
    const bool exact_bm = a.n_terms <= kBmWords * 32;
    const uint32_t* qt = a.tok + a.pos[q];
    const uint32_t send = unsorted ? a.n : a.send[lq];
    if (send <= q + 1) return;
    // 1. stage the query (and its term bitmap); full windows [q+1, send)
    for (uint32_t j = tid; j < lq; j += NT) {
        uint32_t x = __ldg(qt + j);
        qtok[j] = x;
        if (MODE == MODE_FUSED) {
            uint32_t b = exact_bm ? x : ((x * 0x9E3779B1u) >> 16);
            atomicOr(&bm[b >> 5], 1u << (b & 31));
        }
    }
    __syncthreads();
    for (uint32_t j = tid; j < qp; j += NT) {
        uint32_t w = qtok[j];
        uint32_t b = __ldg(a.list_off + w), e = __ldg(a.list_off + w + 1);
        uint32_t lo = lower_bound_src(a.ent, b, e, q + 1);
        uint32_t hi = unsorted ? e : lower_bound_src(a.ent, lo, e, send);
        wlo[j] = lo;
        whi[j] = hi;
    }
    if (tid == 0) {
        s_vc = 0;
        s_cand = 0;
        s_win = 0;
        s_sp = 1;
        s_sa[0] = q + 1;
        s_sb[0] = send;
    }
    // 2. chunks of the id window, depth first
    for (;;) {
        __syncthreads();
        const uint32_t sp = s_sp;
        if (sp == 0) break;
        const uint32_t ra = s_sa[sp - 1], rb = s_sb[sp - 1];
        // windows of this id range and their exclusive scan
        {
            constexpr uint32_t PER = (kPCap + NT - 1) / NT;
            const uint32_t b0 = tid * PER;
            uint32_t loc[PER];
            uint32_t sum = 0;
#pragma unroll
            for (uint32_t i = 0; i < PER; i++) {
                const uint32_t j = b0 + i;
                uint32_t cnt = 0;
                if (j < qp) {
                    const uint32_t lo0 = wlo[j], hi0 = whi[j];
                    const uint32_t lo = (ra == q + 1) ? lo0 : lower_bound_src(a.ent, lo0, hi0, ra);
                    const uint32_t hi = (rb == send) ? hi0 : lower_bound_src(a.ent, lo, hi0, rb);
                    cnt = hi - lo;
                    clo[j] = lo;
                }
                loc[i] = cnt;
                sum += cnt;
            }
            uint32_t tot;
            uint32_t pre = block_excl_scan<uint32_t>(sum, wsum, &tot);
#pragma unroll
            for (uint32_t i = 0; i < PER; i++) {
                const uint32_t j = b0 + i;
                if (j < qp) wpre[j] = pre;
                pre += loc[i];
            }
            if (tid == 0) {
                wpre[qp] = tot;
                s_L = tot;
            }
        }
        __syncthreads();
        const uint32_t L = s_L;
        if (L > Lay::cap && rb - ra > 1) {
            // split the id range; the lower half is processed first
            if (tid == 0) {
                uint32_t mid = ra + (rb - ra) / 2;
                s_sa[sp - 1] = mid;
                s_sb[sp - 1] = rb;
                s_sa[sp] = ra;
                s_sb[sp] = mid;
                s_sp = sp + 1;
            }
            continue;
        }
        if (tid == 0) s_sp = sp - 1;
        if (L == 0) continue;
        if (tid == 0) s_win += L;
        int hl = 6;
        while ((1u << hl) < 2 * L && hl < HLOG) hl++;
        const uint32_t He = 1u << hl, mask = He - 1;
        // 3. accumulate (source, matches, last query position)
        for (uint32_t f = tid; f < L; f += NT) {
            const uint32_t j = upper_bound_gen(wpre, 0, qp, f) - 1;
            const uint32_t k = clo[j] + (f - wpre[j]);
            const uint32_t s = __ldg(&a.ent[k].x);
            if (unsorted && !size_ok(a, lq, a.len[s])) continue;
            if (a.side && __ldg(a.side + s) == __ldg(a.side + q)) continue;
            if (!slot_add(slots, mask, hl, s, j)) atomicOr(a.status, ST_HASH_FULL);
        }
        __syncthreads();
        // 4. per slot: reference candidate? needs a merge?
        uint32_t my_cand = 0, my_ver = 0;
        for (uint32_t h = tid; h < He; h += NT) {
            const unsigned long long v = slots[h];
            const uint32_t s = (uint32_t)(v >> 32);
            if (s == kEmpty) continue;
            const uint32_t c = ((uint32_t)v >> 16) & 0xffffu, jm = (uint32_t)v & 0xffffu;
            const SlotVerdict vd = slot_verdict(a, lq, c, jm, s, qtok[jm]);
            my_cand += vd.cand;
            if (vd.ver) {
                my_ver++;
                if (MODE == MODE_FILL) {
                    uint32_t i = atomicAdd(&s_vc, 1u);
                    if (i < a.vcnt[q]) a.cand[a.voff[q] + i] = make_uint4(q, s, c, jm);
                    else atomicOr(a.status, ST_HASH_FULL);
                } else if (MODE == MODE_FUSED) {
                    // 5. merge right here, one thread per candidate, against the query bitmap
                    const uint32_t ls = a.len[s], S = lq + ls;
                    const uint32_t im = a.inter_min[S];
                    uint32_t nread = 0;
                    const uint32_t o = thread_merge(a.tok + a.pos[s], c, ls, qtok[jm], c, lq - jm - 1, im, bm,
                                                    exact_bm, qtok, jm + 1, lq, &nread);
                    ctr.verified++;
                    ctr.merged += nread;
                    if (o >= im && o > 0) {
                        ctr.inter++;
                        if (o >= a.need[S]) {
                            ctr.res++;
                            emit_result(a, q, s, o);
                        }
                    }
                }
            }
        }
        my_cand = warp_sum(my_cand);
        my_ver = warp_sum(my_ver);
        if (lane == 0) {
            if (my_cand) atomicAdd(&s_cand, my_cand);
            if (MODE == MODE_COUNT && my_ver) atomicAdd(&s_vc, my_ver);
        }
        __syncthreads();
        // 6. clear the slots of this chunk
        for (uint32_t h = tid; h < He; h += NT) slots[h] = kEmptySlot;
    }
    __syncthreads();
    if (tid == 0) {
        if (MODE == MODE_COUNT) {
            a.vcnt[q] = s_vc;
            a.ccnt[q] = s_cand;
            a.wcnt[q] = s_win;
        } else if (MODE == MODE_FUSED) {
            ctr.cand += s_cand;
            ctr.window += s_win;
        }
    }
    if (MODE == MODE_FUSED) {
        for (uint32_t j = tid; j < lq; j += NT) {
            uint32_t x = qtok[j];
            uint32_t b = exact_bm ? x : ((x * 0x9E3779B1u) >> 16);
            bm[b >> 5] = 0u;
        }
    }
    __syncthreads();
}

// Light-query kernel.  items == nullptr: one CTA per query of joins[0]
// (plain method).  Otherwise persistent: CTAs pull (join, q_begin, q_end)
// items from a queue.
template <int MODE, int NT, int HLOG>
__global__ void __launch_bounds__(NT) k_probe(const JoinArgs* __restrict__ joins, const uint4* __restrict__ items,
                                              uint32_t n_items, uint32_t* item_counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    using Lay = ProbeLayout<MODE, HLOG>;
    unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem);
    for (uint32_t h = threadIdx.x; h < Lay::H; h += NT) slots[h] = kEmptySlot;
    if (MODE == MODE_FUSED) {
        uint32_t* bm = reinterpret_cast<uint32_t*>(smem + Lay::off_bm);
        for (uint32_t i = threadIdx.x; i < kBmWords; i += NT) bm[i] = 0u;
    }
    __syncthreads();
    CtaCounters ctr = {0, 0, 0, 0, 0, 0, 0};
    if (items == nullptr) {
        const JoinArgs& a = joins[0];
        probe_query_smem<MODE, NT, HLOG>(a, blockIdx.x, smem, ctr);
        if (MODE == MODE_FUSED) flush_counters_warp(a, ctr);
        return;
    }
    __shared__ uint32_t s_item;
    uint32_t cur_join = 0xffffffffu;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(item_counter, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        __syncthreads();
        if (it >= n_items) break;
        const uint4 w = items[it];
        if (w.x != cur_join) {
            if (cur_join != 0xffffffffu) flush_counters_warp(joins[cur_join], ctr);
            ctr = {0, 0, 0, 0, 0, 0, 0};
            cur_join = w.x;
        }
        const JoinArgs& a = joins[w.x];
        for (uint32_t q = w.y; q < w.z; q++) probe_query_smem<MODE, NT, HLOG>(a, q, smem, ctr);
    }
    if (cur_join != 0xffffffffu) flush_counters_warp(joins[cur_join], ctr);
}

// ------------------------------------------------------------ heavy queries

// Queries past the shared-memory caps (long records): a per-CTA dense
// accumulator in global memory, slot = source id.  The entries' source
// positions give the exact last match directly.
// Scratch per CTA slot: `zero` holds the per-source counters gcnt, gmp (n
// words each), all zero between queries (zeroed once when allocated; every
// query clears the sources it touched), in a buffer of their own so that no
// other array, whatever its layout for another join, ever dirties them;
// `aux` holds the touched and verify lists and the query's windows.
// Joins [join_id, join_id + n_join) one after another, each with its own
// queue counter (queue_counter[j - join_id]); the scratch is sized for the
// largest of them.  Each round of NT joins first lists, in join order, the
// ones with deferred queries, so a batch of joins without any costs one pass.
template <int MODE, int NT>
__global__ void __launch_bounds__(NT) k_probe_heavy(const JoinArgs* __restrict__ joins, uint32_t join_id,
                                                    uint32_t n_join, uint32_t* __restrict__ zero, uint64_t zero_words,
                                                    uint32_t* __restrict__ aux, uint64_t aux_words,
                                                    uint32_t* queue_counter) {
    __shared__ uint32_t s_item, s_nt, s_nv, s_tot, s_nc;
    __shared__ uint32_t wsum[33];
    __shared__ uint32_t s_act[NT];
    for (uint32_t round = 0; round < n_join; round += NT) {
        __syncthreads();  // every thread is done with the previous round's list
        uint32_t nact;
        {
            const uint32_t jr = round + threadIdx.x;
            const uint32_t has = (jr < n_join && *joins[join_id + jr].heavy_count > 0) ? 1u : 0u;
            const uint32_t at = block_excl_scan<uint32_t>(has, wsum, &nact);
            if (has) s_act[at] = jr;
        }
        __syncthreads();
        for (uint32_t x = 0; x < nact; x++) {
            __syncthreads();  // every thread is done with the previous join's queue
            const uint32_t jj = s_act[x];
            const JoinArgs& a = joins[join_id + jj];
            const uint32_t n = a.n;
            uint32_t* gcnt = zero + (uint64_t)blockIdx.x * zero_words;
            uint32_t* gmp = gcnt + n;
            uint32_t* base = aux + (uint64_t)blockIdx.x * aux_words;
            uint32_t* gtouch = base;
            uint32_t* gver = base + (uint64_t)n;
            uint32_t* wlo = base + 2 * (uint64_t)n;
            uint32_t* wpre = wlo + 65536;
            const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
            constexpr uint32_t NW = NT / 32;
            CtaCounters ctr = {0, 0, 0, 0, 0, 0, 0};
            const uint32_t nheavy = min(*a.heavy_count, a.heavy_cap);
            const bool unsorted = (*a.status & ST_UNSORTED) != 0;
            for (;;) {
                if (tid == 0) {
                    s_item = atomicAdd(queue_counter + jj, 1u);
                    s_nt = 0;
                    s_nv = 0;
                    s_nc = 0;
                }
                __syncthreads();
                const uint32_t it = s_item;
                if (it >= nheavy) break;
                const uint32_t q = a.heavy_q[it];
                const uint32_t lq = a.len[q];
                const uint32_t* qt = a.tok + a.pos[q];
                const uint32_t qp = a.probe[lq];
                const uint32_t send = unsorted ? n : a.send[lq];
                for (uint32_t j = tid; j < qp; j += NT) {
                    uint32_t w = __ldg(qt + j);
                    uint32_t b = __ldg(a.list_off + w), e = __ldg(a.list_off + w + 1);
                    uint32_t lo = lower_bound_src(a.ent, b, e, q + 1);
                    uint32_t hi = unsorted ? e : lower_bound_src(a.ent, lo, e, max(send, q + 1));
                    wlo[j] = lo;
                    wpre[j] = hi - lo;
                }
                __syncthreads();
                uint32_t carry = 0;
                for (uint32_t b0 = 0; b0 < qp; b0 += NT) {
                    uint32_t j = b0 + tid;
                    uint32_t x = j < qp ? wpre[j] : 0;
                    uint32_t tot;
                    uint32_t pre = block_excl_scan<uint32_t>(x, wsum, &tot);
                    if (j < qp) wpre[j] = pre + carry;
                    carry += tot;
                }
                if (tid == 0) {
                    wpre[qp] = carry;
                    s_tot = carry;
                }
                __syncthreads();
                const uint32_t L = s_tot;
                if (tid == 0) {
                    ctr.window += L;
                    ctr.heavy++;
                }
                for (uint32_t f = tid; f < L; f += NT) {
                    uint32_t j = upper_bound_gen(wpre, 0, qp, f) - 1;
                    uint32_t k = wlo[j] + (f - wpre[j]);
                    const uint2 e = __ldg(a.ent + k);
                    uint32_t s = e.x;
                    uint32_t sp = e.y & 0xffffu;
                    if (unsorted && !size_ok(a, lq, a.len[s])) continue;
                    if (a.side && __ldg(a.side + s) == __ldg(a.side + q)) continue;
                    uint32_t old = atomicAdd(&gcnt[s], 1u);
                    if (old == 0) gtouch[atomicAdd(&s_nt, 1u)] = s;
                    atomicMax(&gmp[s], (j << 16) | sp);
                }
                __syncthreads();
                const uint32_t nt = s_nt;
                uint32_t my_cand = 0;
                for (uint32_t i = tid; i < nt; i += NT) {
                    uint32_t s = gtouch[i];
                    uint32_t c = gcnt[s], m = gmp[s];
                    uint32_t jm = m >> 16, smx = m & 0xffffu;
                    uint32_t ls = a.len[s], S = lq + ls;
                    uint32_t ub1 = c + min(lq - jm, ls - smx);
                    if (ub1 >= a.cand_min[S]) my_cand++;
                    if (ub1 - 1 >= a.inter_min[S]) {
                        uint32_t v = atomicAdd(&s_nv, 1u);
                        if (MODE == MODE_FILL) {
                            if (v < a.vcnt[q]) a.cand[a.voff[q] + v] = make_uint4(q, s, c, jm);
                            else atomicOr(a.status, ST_HASH_FULL);
                        }
                        else if (MODE == MODE_FUSED) gver[v] = s;
                    }
                }
                my_cand = warp_sum(my_cand);
                if (lane == 0 && my_cand) atomicAdd(&s_nc, my_cand);
                __syncthreads();
                const uint32_t nv = s_nv;
                if (MODE == MODE_COUNT) {
                    if (tid == 0) {
                        a.vcnt[q] = nv;
                        a.ccnt[q] = s_nc;
                        a.wcnt[q] = L;
                    }
                } else if (MODE == MODE_FUSED) {
                    if (tid == 0) ctr.cand += s_nc;
                    for (uint32_t v = wid; v < nv; v += NW) {
                        uint32_t s = gver[v];
                        uint32_t c = gcnt[s], m = gmp[s];
                        uint32_t jm = m >> 16, smx = m & 0xffffu;
                        uint32_t ls = a.len[s], S = lq + ls;
                        uint32_t imin = a.inter_min[S];
                        uint32_t o = warp_merge_count(qt, jm + 1, lq, a.tok + a.pos[s], smx + 1, ls, c, imin);
                        if (lane == 0) {
                            ctr.verified++;
                            if (o >= imin && o > 0) {
                                ctr.inter++;
                                if (o >= a.need[S]) {
                                    ctr.res++;
                                    emit_result(a, q, s, o);
                                }
                            }
                        }
                    }
                }
                __syncthreads();
                for (uint32_t i = tid; i < nt; i += NT) {
                    uint32_t s = gtouch[i];
                    gcnt[s] = 0;
                    gmp[s] = 0;
                }
                __syncthreads();
            }
            if (lane == 0) {
                if (MODE == MODE_FUSED) flush_counters(a, ctr);
                else if (MODE == MODE_COUNT && tid == 0 && ctr.heavy) atomicAdd(&a.stats[SS_HEAVY], ctr.heavy);
            }
        }
    }
}

// Bitmap filter (the bitwise overlap bound of Sandes, Teodoro and Melo for
// exact set similarity joins): every record's tokens hashed into a bitmap.  A
// bit set in only one of two bitmaps comes from at least one token in only one
// of the two records, so |x & y| <= (|x| + |y| - popcount(b(x) ^ b(y))) / 2.
// Warp per record (a long record's bitmap is nearly full and bounds little,
// but it is exact, so the bound holds for every pair).  Width: bmw uint4 per
// record, 2 (256 bits) or 4 (512 bits, for joins of longer records).
// One record's bitmap (warp-collective); sw: the warp's 16 shared words.
__device__ __forceinline__ void bitmap_record(const JoinArgs& a, uint32_t r, uint4* __restrict__ bmap, uint32_t bmw,
                                              uint32_t* sw) {
    const uint32_t lane = lane_id();
    const uint32_t shift = bmw == 4 ? 23 : 24;  // bit index: top 9 or 8 bits of a multiplicative hash
    if (lane < 16) sw[lane] = 0;
    __syncwarp();
    const uint32_t l = a.len[r];
    const uint32_t* t = a.tok + a.pos[r];
    for (uint32_t j = lane; j < l; j += 32) {
        const uint32_t b = (__ldg(t + j) * 0x9E3779B1u) >> shift;
        atomicOr(&sw[b >> 5], 1u << (b & 31));
    }
    __syncwarp();
    if (lane < bmw)
        bmap[(uint64_t)bmw * r + lane] = make_uint4(sw[4 * lane], sw[4 * lane + 1], sw[4 * lane + 2], sw[4 * lane + 3]);
    __syncwarp();
}

static __global__ void k_bitmaps(JoinArgs a, uint4* __restrict__ bmap, uint32_t bmw) {
    __shared__ uint32_t sw[8][16];  // launched with 256 threads: a bitmap per warp
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < a.n; r += warps)
        bitmap_record(a, r, bmap, bmw, sw[threadIdx.x >> 5]);
}

// Bitmap width of a join in uint4 words: 4 (512 bits) when its records average
// more than 96 tokens (a 256-bit bitmap of a long record is too full to bound
// much), else 2 (256 bits).
inline uint32_t bitmap_words(uint64_t n_tokens, uint64_t n_sets) {
    return n_tokens > 96ull * (n_sets ? n_sets : 1) ? 4u : 2u;
}

__device__ __forceinline__ uint32_t popc_xor(uint4 a, uint4 b) {
    return __popc(a.x ^ b.x) + __popc(a.y ^ b.y) + __popc(a.z ^ b.z) + __popc(a.w ^ b.w);
}

// ------------------------------------------------- plain verification stage

// Warp per candidate record (q, s, matches, last query position); the source
// position is found by a search, q tokens are searched in global memory.
// Writes the overlap (0 when it cannot reach floor(min overlap)).
// A candidate whose bitmap bound (k_bitmaps) is below floor(min overlap) can
// be no intersection and skips its merge, as in the batched method's kernel.
static __global__ void k_verify(JoinArgs a, const uint4* __restrict__ cand, const uint64_t* __restrict__ d_nc,
                                uint32_t* __restrict__ ov, const uint4* __restrict__ bmap, uint32_t bmw) {
    const uint32_t nc = (uint32_t)*d_nc;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    unsigned long long inter = 0, ver = 0;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nc; i += warps) {
        const uint4 r = cand[i];
        const uint32_t q = r.x, s = r.y, c = r.z, jm = r.w;
        const uint32_t lq = a.len[q], ls = a.len[s], S = lq + ls;
        const uint32_t imin = a.inter_min[S];
        // lanes 0..bmw-1 each xor one 128-bit word of the two bitmaps
        uint32_t pc = lane < bmw ? popc_xor(__ldg(bmap + bmw * q + lane), __ldg(bmap + bmw * s + lane)) : 0u;
        pc = warp_sum(pc);
        uint32_t o = 0;
        if (S >= 2 * imin + pc) {
            const uint32_t* qt = a.tok + a.pos[q];
            const uint32_t* st = a.tok + a.pos[s];
            const uint32_t smx = warp_find(st, a.index[ls], __ldg(qt + jm));
            o = warp_merge_count(qt, jm + 1, lq, st, smx + 1, ls, c, imin);
        }
        const bool ok = o >= imin && o > 0;
        if (lane == 0) {
            ov[i] = ok ? o : 0;
            ver++;
            inter += ok;
        }
    }
    if (lane == 0) {
        if (inter) atomicAdd(&a.stats[SS_INTERSECTIONS], inter);
        if (ver) atomicAdd(&a.stats[SS_VERIFIED], ver);
    }
}

// Result flags for the compaction (block.cu:190-192 as an integer test).
static __global__ void k_result_flags(JoinArgs a, const uint4* __restrict__ cand, const uint32_t* __restrict__ ov,
                               const uint64_t* __restrict__ d_nc, uint32_t* __restrict__ flag) {
    const uint32_t nc = (uint32_t)*d_nc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        uint4 r = cand[i];
        uint32_t S = a.len[r.x] + a.len[r.y];
        uint32_t o = ov[i];
        flag[i] = (o > 0 && o >= a.need[S]) ? 1u : 0u;
    }
}

static __global__ void k_result_fill(const uint4* __restrict__ cand, const uint32_t* __restrict__ ov,
                              const uint32_t* __restrict__ flag, const uint32_t* __restrict__ off,
                              const uint64_t* __restrict__ d_nc, uint64_t* __restrict__ key,
                              uint32_t* __restrict__ val) {
    const uint32_t nc = (uint32_t)*d_nc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        if (flag[i]) {
            uint4 r = cand[i];
            uint32_t d = off[i];
            key[d] = ((uint64_t)r.x << 32) | r.y;
            val[d] = ov[i];
        }
    }
}

// Fused method: results (q, s, o) -> sort keys.
static __global__ void k_result_keys(const uint32_t* __restrict__ rq, const uint32_t* __restrict__ rs,
                              const uint32_t* __restrict__ ro, const uint32_t* __restrict__ d_cnt, uint32_t cap,
                              uint64_t* __restrict__ key, uint32_t* __restrict__ val, uint64_t* __restrict__ d_n) {
    const uint32_t n = min(*d_cnt, cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_n = n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        key[i] = ((uint64_t)rq[i] << 32) | rs[i];
        val[i] = ro[i];
    }
}

// Sorted keys -> output columns: q, s, id_q, id_s, overlap, sim.
static __global__ void k_result_out(const uint64_t* __restrict__ key, const uint32_t* __restrict__ val,
                             const uint64_t* __restrict__ d_n, const uint32_t* __restrict__ id,
                             const uint32_t* __restrict__ len, uint32_t* __restrict__ oq, uint32_t* __restrict__ os,
                             uint32_t* __restrict__ oidq, uint32_t* __restrict__ oids, uint32_t* __restrict__ oo,
                             float* __restrict__ osim) {
    const uint64_t n = *d_n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = key[i];
        uint32_t q = (uint32_t)(k >> 32), s = (uint32_t)k, o = val[i];
        oq[i] = q;
        os[i] = s;
        oidq[i] = id ? id[q] : q;
        oids[i] = id ? id[s] : s;
        oo[i] = o;
        uint32_t uni = len[q] + len[s] - o;
        osim[i] = __fdiv_rn(__uint2float_rn(o), __uint2float_rn(uni));  // similarity.cuh:78-82
    }
}

}  // namespace fgss
