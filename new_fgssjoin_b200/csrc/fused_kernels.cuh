// fused_kernels.cuh -- the batched method's filter + verify kernel.
//
// Same semantics as the plain stages (join_kernels.cuh; reference
// filtering.cu:76-141, checking.cu:93-175, block.cu:184-197), organised for
// throughput:
//   * windows_query: one warp per query computes the id window [q+1, send)
//     of every probe token's list by binary search, the prefix of the window
//     sizes and the per-query total that sizes work items (launched for every
//     join of a batch at once by k_windows_mj, batch_kernels.cuh).
//   * chunks_query: queries whose windows hold more entries than 3/4 of the
//     slot table get precomputed id-range chunk boundaries (k_chunks_mj).
//   * bitmap_record: a token bitmap per record (the bitmap filter, k_bitmaps_mj).
//   * k_fused: persistent CTAs pull work items (runs of queries of one join,
//     longest first, claimed one item ahead).  Per query: the query's tokens
//     and a membership structure (bitmap, hashed set or hashed bitmap) go to
//     shared memory; per chunk of its id window the window entries are
//     accumulated into a shared-memory slot table (64-bit CAS per entry; the
//     index entry carries the source's size), the occupied slots are decided
//     from shared memory and L1 alone, the deciding lane checks the bitmap
//     bound of the survivors, and warps merge the few that remain.
#pragma once

#include "join_kernels.cuh"

namespace fgss {

// Slot word: source id (32) | query position of the last match (11) |
// source position of the last match (11; 2047 = too large to keep) |
// number of prefix matches (10).
constexpr uint32_t kSmaxUnknown = 2047;

// The query's membership structure (bitmap, hashed set or hashed bitmap): 2^kMemberBits bits.
constexpr uint32_t kMemberBits = 14;
constexpr uint32_t kMemberWords = 1u << (kMemberBits - 5);

// Layout: slots u64[H] | occ u32[cap] | cbr u32[PC] | jr u16[PC] |
//         sbits u32[JW] | gpre u16[JW] | qtok u32[QC] | bm u32[BW] | mlist u32[MC]
// occ and mlist entries are slot | source size << 16 (a part's distinct sources
// number at most cap).
// The current part's windows are kept in rank form: its non-empty windows in
// order get ranks r, cbr[r] = first entry - entries of the earlier windows
// (so entry f of the part is ent[cbr[r] + f]) and jr[r] = the probe position;
// bit f of sbits is set where a window starts, gpre[g] = windows starting
// before entry 32 g.  Entry f's window is then rank gpre[f / 32] - 1 plus the
// starts at or below f in its group: two broadcast loads and a popcount.
template <int HLOG>
struct FusedLayout {
    static constexpr uint32_t H = 1u << HLOG;
    static constexpr uint32_t cap = H / 4 * 3;  // window entries per chunk (load <= 3/4)
    // probe tokens handled in shared memory: 256..384 (a slot's 11-bit query
    // position and 10-bit match count rely on PC <= 512); a query with more
    // goes to the global-memory accumulator.  The staging caps keep the
    // 2^11-slot layout at 30 KB, 7 CTAs of 128 threads per SM
    static constexpr uint32_t PC = H / 4 > 384 ? 384 : (H / 4 > 256 ? H / 4 : 256);
    static constexpr uint32_t QC = H / 2 > 512 ? 512 : H / 2;  // query tokens staged in shared memory
                                                                  // (longer: read from HBM)
    // entries of one part: at most cap, or PC when a part of one source id
    // (which holds at most one entry per probe window) cannot be bisected
    static constexpr uint32_t JE = cap > PC ? cap : PC;
    static constexpr uint32_t JW = (JE + 31) / 32;  // groups of 32 entries
    static constexpr uint32_t BW = kMemberWords;  // membership words: 16384 bits
    static constexpr uint32_t MC = 256;       // merge list entries per chunk (more: merged by their lane)
    static constexpr size_t al16(size_t x) { return (x + 15) & ~size_t(15); }
    static constexpr size_t off_occ = 8ull * H;
    static constexpr size_t off_cbr = off_occ + 4ull * cap;
    static constexpr size_t off_jr = off_cbr + 4ull * PC;
    static constexpr size_t off_sbits = al16(off_jr + 2ull * PC);
    static constexpr size_t off_gpre = off_sbits + 4ull * JW;
    static constexpr size_t off_qtok = al16(off_gpre + 2ull * JW);
    static constexpr size_t off_bm = off_qtok + 4ull * QC;
    static constexpr size_t off_ml = off_bm + 4ull * BW;
    static constexpr size_t bytes = off_ml + 4ull * MC;
    static_assert(off_bm % 16 == 0, "the membership words are cleared with 16-byte stores");
};

// Windows of one query's probe tokens (warp-collective): win[poff[q] + j] =
// (lo, hi), wpre[poff[q] + j] = entries in the query's windows before window j,
// wtot[q] = sum of the window sizes (also meta[q].w).
__device__ __forceinline__ void windows_query(const JoinArgs& a, uint32_t q, const uint32_t* __restrict__ poff,
                                              uint2* __restrict__ win, uint32_t* __restrict__ wpre,
                                              uint32_t* __restrict__ wtot, uint4* __restrict__ meta) {
    const uint32_t lane = lane_id();
    const bool unsorted = (*a.status & ST_UNSORTED) != 0;
    const uint32_t lq = a.len[q];
    const bool mine = q >= a.q_lo && q < a.q_hi;
    const uint32_t qp = (lq <= 65535u && mine) ? a.probe[lq] : 0;
    const uint32_t send = unsorted ? a.n : (lq <= 65535u ? a.send[lq] : 0);
    const uint32_t* qt = a.tok + a.pos[q];
    const uint32_t o = poff[q];
    uint32_t tot = 0;  // running total of the windows before this round (same in every lane)
    for (uint32_t j0 = 0; j0 < qp; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t lo = 0, hi = 0;
        if (j < qp) {
            const uint32_t w = __ldg(qt + j);
            const uint32_t b = __ldg(a.list_off + w), e = __ldg(a.list_off + w + 1);
            lo = e;
            hi = e;
            if (send > q + 1) {
                lo = lower_bound_src(a.ent, b, e, q + 1);
                hi = unsorted ? e : lower_bound_src(a.ent, lo, e, send);
            }
        }
        const uint32_t incl = warp_incl_scan(hi - lo);
        if (j < qp) {
            win[o + j] = make_uint2(lo, hi);
            wpre[o + j] = tot + incl - (hi - lo);
        }
        tot += __shfl_sync(kFull, incl, 31);
    }
    if (lane == 0) {
        wtot[q] = tot;
        meta[q] = make_uint4(a.pos[q], lq, lq <= 65535u ? a.index[lq] : 0u, tot);
    }
}

// Chunks of one query's id window [q+1, send) whose windows hold L entries:
// 1 when they fit `cap`, else enough equal id ranges for 3/4 of cap on
// average (at most one per id).  Also gives the probe prefix and the span.
__device__ __forceinline__ uint32_t chunk_count(const JoinArgs& a, uint32_t q, uint32_t L, uint32_t cap, uint32_t& qp,
                                                uint32_t& span) {
    const bool unsorted = (*a.status & ST_UNSORTED) != 0;
    const uint32_t lq = a.len[q];
    qp = lq <= 65535u ? a.probe[lq] : 0;
    const uint32_t send = unsorted ? a.n : (lq <= 65535u ? a.send[lq] : 0);
    span = send > q + 1 ? send - q - 1 : 0;
    if (L <= cap || qp == 0 || send <= q + 2) return 1;
    const uint64_t want = ((uint64_t)L * 4 + 3ull * cap - 1) / (3ull * cap);
    return (uint32_t)(want < span ? want : span);
}

// Chunk boundaries of one query whose windows hold more than `cap` entries
// (warp-collective): the id window [q+1, send) is cut into nch equal id ranges
// (sized for 3/4 of cap on average) and, for every inner boundary id b and
// probe token j, the first entry of j's window at or after b is stored.  The
// boundary buffer is carved with one atomic per query; a query that does not
// fit keeps nch = 1 and the fused kernel bisects it instead.
__device__ __forceinline__ void chunks_query(const JoinArgs& a, uint32_t q, const uint32_t* __restrict__ poff,
                                             const uint2* __restrict__ win, const uint32_t* __restrict__ wtot,
                                             uint32_t cap, uint2* __restrict__ qchunk, uint32_t* __restrict__ cbuf,
                                             uint64_t cbuf_cap, unsigned long long* __restrict__ cbuf_used) {
    const uint32_t lane = lane_id();
    uint32_t qp, span;
    uint32_t nch = chunk_count(a, q, wtot[q], cap, qp, span);
    unsigned long long base = 0;
    if (nch > 1) {
        if (lane == 0) {
            const unsigned long long need = (unsigned long long)(nch - 1) * qp;
            base = atomicAdd(cbuf_used, need);
            if (base + need > cbuf_cap) nch = 1;
        }
        nch = __shfl_sync(kFull, nch, 0);
        base = __shfl_sync(kFull, base, 0);
        if (nch > 1) {
            const uint2* w = win + poff[q];
            const uint32_t inner = (nch - 1) * qp;
            for (uint32_t f = lane; f < inner; f += 32) {
                const uint32_t i = f / qp + 1, j = f % qp;
                const uint32_t b = q + 1 + (uint32_t)(((uint64_t)span * i) / nch);
                const uint2 wj = w[j];
                cbuf[base + f] = lower_bound_src(a.ent, wj.x, wj.y, b);
            }
        }
    }
    if (lane == 0) qchunk[q] = make_uint2((uint32_t)base, nch);
}

struct FusedArgs {
    const uint32_t* poff;    // per query: first probe window
    const uint2* win;
    const uint4* smin;       // per length sum S: (cand_min, inter_min, need, 0)
    const uint4* meta;       // per record: (pos, len, index prefix, window entries)
    const uint32_t* wpre;    // per probe window: entries of the query's earlier windows
    const uint2* qchunk;     // per query: (first boundary in cbuf, number of chunks)
    const uint32_t* cbuf;    // chunk boundaries: per inner boundary, first entry of each probe window
    const uint4* bmap;       // per record: token bitmap of bmw uint4
    uint32_t bmw;            // 2 (256 bits) or 4 (512 bits)
};

// Query-token membership, three forms chosen per query (the same for every
// thread of the CTA):
//   QM_EXACT  vocabulary of at most 2^kMemberBits terms: one bit per term;
//   QM_HASH   larger vocabulary, query of at most kQHashMax tokens: open-addressing
//             set of token + 1 in the same kMemberWords words (load <= 1/2, 0 = empty);
//   QM_BLOOM  otherwise: one bit per hash, hits confirmed by binary search.
enum : uint32_t { QM_EXACT = 0, QM_HASH = 1, QM_BLOOM = 2 };
constexpr uint32_t kQHashBits = kMemberBits - 5, kQHashWords = 1u << kQHashBits, kQHashMax = kQHashWords / 2;

// Start slot of token x in the hashed set; bit of x in the hashed bitmap.
__device__ __forceinline__ uint32_t qhash(uint32_t x) { return (x * 0x9E3779B1u) >> (32 - kQHashBits); }
__device__ __forceinline__ uint32_t bloom_bit(uint32_t x) { return (x * 0x9E3779B1u) >> (32 - kMemberBits); }

__device__ __forceinline__ bool bm_test(const uint32_t* bm, uint32_t mode, uint32_t x, const uint32_t* qtok,
                                        uint32_t qa, uint32_t lq) {
    if (mode == QM_HASH) {
        uint32_t h = qhash(x);
        for (uint32_t it = 0; it < kQHashWords; it++) {
            const uint32_t v = bm[h];
            if (v == x + 1u) return true;
            if (v == 0u) return false;
            h = (h + 1u) & (kQHashWords - 1u);
        }
        return false;
    }
    const uint32_t b = mode == QM_EXACT ? x : bloom_bit(x);
    bool hit = (bm[b >> 5] >> (b & 31)) & 1u;
    if (hit && mode != QM_EXACT) hit = contains_gen(qtok, qa, lq, x);
    return hit;
}

// Puts query token x into the membership structure of the chosen form.
__device__ __forceinline__ void bm_insert(uint32_t* bm, uint32_t mode, uint32_t x) {
    if (mode == QM_HASH) {
        uint32_t h = qhash(x);
        for (uint32_t it = 0; it < kQHashWords; it++) {
            const uint32_t prev = atomicCAS(&bm[h], 0u, x + 1u);
            if (prev == 0u || prev == x + 1u) return;
            h = (h + 1u) & (kQHashWords - 1u);
        }
        return;
    }
    const uint32_t b = mode == QM_EXACT ? x : bloom_bit(x);
    atomicOr(&bm[b >> 5], 1u << (b & 31));
}

// The fused kernel's per-thread counters, 32-bit to keep registers free; they
// are added to the join's 64-bit statistics when the CTA moves to another join
// (or one of them passes 2^30) and at the end.
struct FusedCounters {
    uint32_t cand, inter, res, window, verified, merged, qtok;
};

// Warp-collective: adds the warp's counters to the join's statistics and clears them.
__device__ __forceinline__ void flush_fused_counters(const JoinArgs& a, FusedCounters& c) {
    const unsigned long long v[7] = {warp_sum((unsigned long long)c.cand), warp_sum((unsigned long long)c.inter),
                                     warp_sum((unsigned long long)c.res), warp_sum((unsigned long long)c.window),
                                     warp_sum((unsigned long long)c.verified), warp_sum((unsigned long long)c.merged),
                                     warp_sum((unsigned long long)c.qtok)};
    if (lane_id() == 0) {
        const int idx[7] = {SS_CANDIDATES, SS_INTERSECTIONS, SS_RESULTS, SS_WINDOW, SS_VERIFIED, SS_MERGED, SS_QTOK};
#pragma unroll
        for (int i = 0; i < 7; i++)
            if (v[i]) atomicAdd(&a.stats[idx[i]], v[i]);
    }
    c = {0, 0, 0, 0, 0, 0, 0};
}

// One merge step: up to 8 source tokens from position k (two independent
// 16-byte loads of the aligned chunks holding them; the second only when it
// holds tokens of this record, so no load leaves the record's 16-byte blocks).
__device__ __forceinline__ uint32_t merge_step(const uint32_t* __restrict__ st, uint32_t& k, uint32_t ls,
                                               uint32_t xq, const uint32_t* bm, uint32_t mode, const uint32_t* qt,
                                               uint32_t lq) {
    const uintptr_t addr = reinterpret_cast<uintptr_t>(st + k);
    const uint4* p = reinterpret_cast<const uint4*>(addr & ~uintptr_t(15));
    const uint32_t off = (uint32_t)(addr & 15u) >> 2;
    const uint32_t avail = ls - k;  // >= 1
    const uint4 v0 = __ldg(p);
    const bool two = avail > 4u - off;
    uint4 v1 = make_uint4(0, 0, 0, 0);
    if (two) v1 = __ldg(p + 1);
    const uint32_t n_in = min(8u - off, avail);
    const uint32_t xs[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
    uint32_t hits = 0;
#pragma unroll
    for (uint32_t t = 0; t < 8; t++) {
        if (t >= off && t < off + n_in) {
            const uint32_t x = xs[t];
            if (x > xq && bm_test(bm, mode, x, qt, 0, lq)) hits++;
        }
    }
    k += n_in;
    return hits;
}

// Counts one candidate whose verification is finished with overlap o.
__device__ __forceinline__ void tally_overlap(const JoinArgs& a, FusedCounters& ctr, uint32_t q, uint32_t s,
                                              uint32_t o, uint32_t im, uint32_t need) {
    if (o >= im && o > 0) {
        ctr.inter++;
        if (o >= need) {
            ctr.res++;
            emit_result(a, q, s, o);
        }
    }
}

// SIDED: an R-S join (a.side set); self-joins use the instantiation without the side test.
//
// Per query: stage its tokens and membership structure, then per chunk of its
// id window (one chunk when the windows fit the slot table):
//   1. accumulate: every window entry (source s, query position j, source
//      position and size from the index entry; its window from the part's
//      rank form) goes into the shared slot table, always used whole, with a
//      read of its slot and one 64-bit CAS (key s; match count, last match
//      positions); a newly occupied slot records the source's size beside it,
//      and the slots a warp's four entry steps newly occupied go onto the
//      occupied list with one shared atomic;
//   2. decide: per occupied slot the reference-candidate and needs-merge tests
//      read the slot word, the size beside it and the bound table (no gather
//      per source); a slot that still needs a merge loads the source's bitmap
//      (2 or 4 16-byte words) and, if the bitmap bound can still reach
//      floor(min overlap), goes on the merge list (one shared atomic per warp);
//   3. merge: warps take the merge list, 32 source tokens per step (one
//      coalesced load, a membership test per lane, ballot + popcount), with
//      the early exit of checking.cu:150-157; slots are cleared meanwhile.
// Every loop that ballots runs per warp (its bound is the same on all lanes).
template <int NT, int HLOG, bool SIDED>
__device__ void fused_query(const JoinArgs& a, const FusedArgs& fa, uint32_t q, unsigned char* smem,
                            FusedCounters& ctr) {
    using Lay = FusedLayout<HLOG>;
    constexpr uint32_t NW = NT / 32;
    unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* occ = reinterpret_cast<uint32_t*>(smem + Lay::off_occ);
    uint32_t* cbr = reinterpret_cast<uint32_t*>(smem + Lay::off_cbr);
    uint16_t* jr = reinterpret_cast<uint16_t*>(smem + Lay::off_jr);
    uint32_t* sbits = reinterpret_cast<uint32_t*>(smem + Lay::off_sbits);
    uint16_t* gpre = reinterpret_cast<uint16_t*>(smem + Lay::off_gpre);
    uint32_t* qtok = reinterpret_cast<uint32_t*>(smem + Lay::off_qtok);
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + Lay::off_bm);
    uint32_t* mlist = reinterpret_cast<uint32_t*>(smem + Lay::off_ml);
    __shared__ uint32_t s_sp, s_nocc, s_nm, s_cand, s_win, s_L;
    __shared__ uint4 s_qbm[4];  // the query's bitmap
    __shared__ uint32_t s_sa[48], s_sb[48], s_sc[48];
    constexpr uint32_t kNoPart = 0xffffffffu, kBisected = 0xfffffffeu;  // s_L: no part left / bisected

    const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t st_bits = *a.status;
    if (st_bits & ST_SKIP_ALL) return;
    if (q < a.q_lo || q >= a.q_hi) return;
    const uint4 qm = fa.meta[q];
    const uint32_t lq = qm.y;
    if (lq == 0 || lq > 65535u) return;
    const uint32_t qp = a.probe[lq];
    if (qp == 0) return;
    const bool unsorted = (st_bits & ST_UNSORTED) != 0;
    const uint32_t send = unsorted ? a.n : a.send[lq];
    if (send <= q + 1) return;
    if (qp > Lay::PC || qp >= a.heavy_min_qp) {  // a query of the global-memory accumulator
        if (tid == 0) defer_heavy(a, q);
        return;
    }
    const uint32_t qmode = a.n_terms <= Lay::BW * 32 ? QM_EXACT : (lq <= kQHashMax ? QM_HASH : QM_BLOOM);
    const uint8_t* sidep = SIDED ? a.side : nullptr;  // R-S join: skip sources on the query's own side
    const uint8_t side_q = SIDED ? __ldg(sidep + q) : 0;
    const uint32_t* qt = a.tok + qm.x;
    const bool staged = lq <= Lay::QC;
    const uint32_t* qsrc = staged ? qtok : qt;  // query tokens: shared memory, or HBM for long records
    const uint2* qwin = fa.win + fa.poff[q];
    const uint2 qc = fa.qchunk[q];
    const uint32_t* cb = fa.cbuf + qc.x;
    const uint32_t nch = qc.y;
    for (uint32_t j = tid; j < lq; j += NT) {
        const uint32_t x = __ldg(qt + j);
        if (staged) qtok[j] = x;
        bm_insert(bm, qmode, x);
    }
    if (tid < fa.bmw) s_qbm[tid] = fa.bmap[fa.bmw * q + tid];
    // one chunk that fits the slot table (the common case): the pre-pass's
    // window prefix is used as is, with no block-wide scan
    const bool one_chunk = nch == 1 && qm.w <= Lay::cap;
    // Warp-collective (warp 0): lays out a part's windows in rank form from
    // bounds(j) = (first entry, end) of probe window j inside the part; returns
    // the part's entries.  A part of more than JE entries is bisected by the
    // caller and its layout never read (starts past JE are not marked).
    auto lay_windows = [&](auto&& bounds) -> uint32_t {
        for (uint32_t g = lane; g < Lay::JW; g += 32) sbits[g] = 0u;
        __syncwarp();
        uint32_t carry = 0, rc = 0;
        for (uint32_t j0 = 0; j0 < qp; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t lo = 0, cnt = 0;
            if (j < qp) {
                const uint2 b = bounds(j);
                lo = b.x;
                cnt = b.y - b.x;
            }
            const uint32_t incl = warp_incl_scan(cnt);
            const uint32_t p = carry + incl - cnt;  // entries of the earlier windows
            const uint32_t nz = __ballot_sync(kFull, cnt != 0);
            if (cnt != 0) {
                const uint32_t r = rc + __popc(nz & lanemask_lt());
                cbr[r] = lo - p;
                jr[r] = (uint16_t)j;
                if (p < Lay::JW * 32) atomicOr(&sbits[p >> 5], 1u << (p & 31));
            }
            carry += __shfl_sync(kFull, incl, 31);
            rc += __popc(nz);
        }
        __syncwarp();
        const uint32_t ng = min((carry + 31) / 32, Lay::JW);
        uint32_t gc = 0;
        for (uint32_t g0 = 0; g0 < ng; g0 += 32) {
            const uint32_t g = g0 + lane;
            const uint32_t c = g < ng ? __popc(sbits[g]) : 0u;
            const uint32_t incl = warp_incl_scan(c);
            if (g < ng) gpre[g] = (uint16_t)(gc + incl - c);
            gc += __shfl_sync(kFull, incl, 31);
        }
        return carry;
    };
    if (one_chunk && wid == 0) lay_windows([&](uint32_t j) { return qwin[j]; });
    if (!one_chunk) {
        // the query's chunk boundaries and windows, into L2 ahead of its part setups
        // (every address stays inside the two arrays)
        const char* b0 = reinterpret_cast<const char*>(cb);
        const uint32_t nb = (nch - 1) * qp * 4u;
        for (uint32_t o = tid * 128u; o < nb; o += NT * 128u) asm volatile("prefetch.global.L2 [%0];" ::"l"(b0 + o));
        if (tid == 0 && nb) asm volatile("prefetch.global.L2 [%0];" ::"l"(b0 + nb - 1));
        const char* w0 = reinterpret_cast<const char*>(qwin);
        for (uint32_t o = tid * 128u; o < qp * 8u; o += NT * 128u) asm volatile("prefetch.global.L2 [%0];" ::"l"(w0 + o));
        if (tid == 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(w0 + qp * 8u - 1));
    }
    if (tid == 0) {
        s_cand = 0;
        s_win = 0;
        s_sp = 0;
        s_nocc = 0;
        s_nm = 0;
        ctr.qtok += lq;
    }
    const uint4* smin = fa.smin + lq;  // indexed by the source size
    // The chunks of the query's id window: a single chunk when its windows fit
    // the slot table, else the precomputed split, whose parts bisect
    // themselves further while they hold more than `cap` entries.  A chunk's
    // windows are laid out in rank form (cbr, jr, sbits, gpre) before it is
    // accumulated, decided and merged.
    const uint32_t span = send - q - 1;
    const uint32_t n_parts = one_chunk ? 1u : nch;
    for (uint32_t ci = 0; ci < n_parts; ci++) {
        __syncthreads();  // the staged query; every thread is done with the chunk stack
        if (tid == 0 && !one_chunk) {
            // chunk ci of the precomputed split (tag ci: windows from the boundary buffer)
            s_sa[0] = q + 1 + (uint32_t)(((uint64_t)span * ci) / nch);
            s_sb[0] = q + 1 + (uint32_t)(((uint64_t)span * (ci + 1)) / nch);
            s_sc[0] = ci;
            s_sp = 1;
        }
        bool single_done = false;
        for (;;) {
            uint32_t L;
            if (one_chunk) {
                if (single_done) break;
                single_done = true;
                L = qm.w;
                if (tid == 0) s_win += L;
            } else {
                __syncthreads();  // the previous part is done with the slots and the windows
                if (wid == 0) {
                    // warp 0: this part's windows and their exclusive prefix, and whether
                    // it must be bisected further (then its halves go on the stack)
                    const uint32_t sp = s_sp;
                    const uint32_t ra = sp ? s_sa[sp - 1] : 0, rb = sp ? s_sb[sp - 1] : 0;
                    const uint32_t tag = sp ? s_sc[sp - 1] : 0;
                    __syncwarp();
                    if (sp == 0) {
                        if (lane == 0) s_L = kNoPart;
                    } else {
                        const uint32_t carry = lay_windows([&](uint32_t j) {
                            if (tag != 0xffffffffu) {
                                const uint32_t lo = tag == 0 ? qwin[j].x : cb[(tag - 1) * qp + j];
                                const uint32_t hi = tag + 1 == nch ? qwin[j].y : cb[tag * qp + j];
                                return make_uint2(lo, hi);
                            }
                            const uint2 wj = qwin[j];
                            const uint32_t lo = lower_bound_src(a.ent, wj.x, wj.y, ra);
                            return make_uint2(lo, lower_bound_src(a.ent, lo, wj.y, rb));
                        });
                        if (lane == 0) {
                            if (carry > Lay::cap && rb - ra > 1) {  // bisect; the lower half first
                                const uint32_t mid = ra + (rb - ra) / 2;
                                s_sa[sp - 1] = mid;
                                s_sb[sp - 1] = rb;
                                s_sc[sp - 1] = 0xffffffffu;
                                s_sa[sp] = ra;
                                s_sb[sp] = mid;
                                s_sc[sp] = 0xffffffffu;
                                s_sp = sp + 1;
                                s_L = kBisected;
                            } else {
                                s_sp = sp - 1;
                                s_win += carry;
                                s_L = carry;
                            }
                        }
                    }
                }
                __syncthreads();  // the part's windows, prefix and fate
                L = s_L;
                if (L == kNoPart) break;
                if (L == kBisected) continue;
            }
            if (L == 0) continue;
            // the whole table for every part: the lowest load, so the shortest probe chains
            const int hl = HLOG;
            const uint32_t mask = (1u << hl) - 1;
            // 1. accumulate: four entries' loads are issued before their slot updates,
            // and the slots they newly occupy go onto the occupied list together.
            // Entries f0 + u NT + lane form one aligned group of 32 per warp.
            for (uint32_t f0 = tid - lane; f0 < L; f0 += 4 * NT) {
                uint32_t sv[4], pv[4], jv[4], clm[4];
#pragma unroll
                for (uint32_t u = 0; u < 4; u++) {
                    const uint32_t g0 = f0 + u * NT, f = g0 + lane;
                    sv[u] = kEmpty;
                    if (f < L) {
                        // the window of entry f: the last one starting at or below f
                        const uint32_t g = g0 >> 5;
                        const uint32_t r = gpre[g] + __popc(sbits[g] & (lanemask_lt() | (1u << lane))) - 1u;
                        const uint2 e = __ldg(a.ent + (cbr[r] + f));  // one 8-byte entry
                        sv[u] = e.x;
                        pv[u] = e.y;  // source size << 16 | source position
                        jv[u] = jr[r];
                    }
                }
#pragma unroll
                for (uint32_t u = 0; u < 4; u++) {
                    const uint32_t s = sv[u];
                    uint32_t claimed = 0xffffffffu;  // the slot this entry newly occupied | size << 16
                    if (s != kEmpty) {
                        const uint32_t ls = pv[u] >> 16;
                        bool skip = unsorted && !size_ok(a, lq, ls);
                        if (SIDED && !skip) skip = __ldg(sidep + s) == side_q;
                        if (!skip) {
                            // query position << 11 | source position (2047: too large to keep)
                            const uint32_t pos = (jv[u] << 11) | min(pv[u] & 0xffffu, kSmaxUnknown);
                            uint32_t h = hash_slot(s, hl);
                            bool done = false;
                            // read the slot first: 1.4 CAS per entry when the first try assumed an empty
                            // slot (every repeat of a source failed once); a read and ~1 CAS this way
                            unsigned long long old = *(volatile unsigned long long*)&slots[h];
                            for (uint32_t it = 0; it <= mask && !done;) {
                                const uint32_t key = (uint32_t)(old >> 32);
                                unsigned long long nw;
                                if (key == s) {
                                    const uint32_t lo = (uint32_t)old;
                                    // positions of later matches are larger on both sides: keep the max
                                    const uint32_t lastpos = max(lo >> 10, pos);
                                    nw = ((unsigned long long)s << 32) | (lastpos << 10) | ((lo & 0x3ffu) + 1u);
                                } else if (key == kEmpty) {
                                    nw = ((unsigned long long)s << 32) | (pos << 10) | 1u;
                                } else {
                                    h = (h + 1) & mask;
                                    it++;
                                    old = *(volatile unsigned long long*)&slots[h];
                                    continue;
                                }
                                const unsigned long long prev = atomicCAS(&slots[h], old, nw);
                                if (prev == old) {
                                    if (key == kEmpty) claimed = h | (ls << 16);
                                    done = true;
                                } else {
                                    old = prev;
                                }
                            }
                            if (!done) atomicOr(a.status, ST_HASH_FULL);
                        }
                    }
                    clm[u] = claimed;
                }
                // the slots the four steps newly occupied onto the occupied list, one shared
                // atomic per warp
                uint32_t mk[4], tot = 0;
#pragma unroll
                for (uint32_t u = 0; u < 4; u++) {
                    mk[u] = __ballot_sync(kFull, clm[u] != 0xffffffffu);
                    tot += __popc(mk[u]);
                }
                if (tot) {
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd(&s_nocc, tot);
                    base = __shfl_sync(kFull, base, 0);
                    const uint32_t lt = lanemask_lt();
#pragma unroll
                    for (uint32_t u = 0; u < 4; u++) {
                        if (clm[u] != 0xffffffffu) occ[base + __popc(mk[u] & lt)] = clm[u];
                        base += __popc(mk[u]);
                    }
                }
            }
            __syncthreads();
            // 2. decide: reference candidate?  needs a merge?  (bitmap bound last)
            const uint32_t nocc = s_nocc;
            uint32_t my_cand = 0;
            for (uint32_t i0 = tid - lane; i0 < nocc; i0 += NT) {
                const uint32_t i = i0 + lane;
                bool check = false;
                uint32_t e = 0;  // slot | source size << 16
                if (i < nocc) {
                    e = occ[i];
                    const uint32_t ls = e >> 16;
                    const uint4 sm = __ldg(smin + ls);  // (cand_min, inter_min, need) of |q| + |s|
                    const unsigned long long v = slots[e & 0xffffu];
                    const uint32_t s = (uint32_t)(v >> 32), lo = (uint32_t)v;
                    const uint32_t c = lo & 0x3ffu, jm = lo >> 21, smx = (lo >> 10) & 0x7ffu;
                    const uint32_t A = lq - jm;
                    bool cand, ver;
                    if (smx != kSmaxUnknown) {
                        // exact last match on both sides (filtering.cu:127-135 at the last match)
                        cand = c + min(A, ls - smx) >= sm.x;
                        ver = c + min(A - 1, ls - smx - 1) >= sm.y;
                    } else {
                        const uint4 sm4 = fa.meta[s];  // (pos, len, index prefix)
                        const uint32_t* st = a.tok + sm4.x;
                        const uint32_t xq = qsrc[jm];
                        cand = (c + A >= sm.x) && smax_le(st, (int)ls + (int)c - (int)sm.x, c, sm4.z, xq);
                        ver = (c + A - 1 >= sm.y) && smax_le(st, (int)ls + (int)c - 1 - (int)sm.y, c, sm4.z, xq);
                    }
                    my_cand += cand;
                    if (ver) {
                        ctr.verified++;
                        // the merge resumes right after the last match (or at c when its position
                        // was not kept); when nothing left can change the count, c is the overlap
                        const uint32_t k = smx != kSmaxUnknown ? smx + 1 : c;
                        if (k >= ls || c + min(ls - k, A - 1) < sm.y) {
                            tally_overlap(a, ctr, q, s, c, sm.y, sm.z);
                        } else {
                            // bitmap bound on the whole overlap: below floor(min overlap), no merge
                            const uint4* b4 = fa.bmap + fa.bmw * s;
                            uint32_t pc = popc_xor(s_qbm[0], __ldg(b4)) + popc_xor(s_qbm[1], __ldg(b4 + 1));
                            if (fa.bmw == 4) pc += popc_xor(s_qbm[2], __ldg(b4 + 2)) + popc_xor(s_qbm[3], __ldg(b4 + 3));
                            check = lq + ls >= 2 * sm.y + pc;
                        }
                    }
                }
                const uint32_t m = __ballot_sync(kFull, check);
                if (m) {  // onto the merge list
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd(&s_nm, (uint32_t)__popc(m));
                    base = __shfl_sync(kFull, base, 0);
                    if (check) {
                        const uint32_t mi = base + __popc(m & lanemask_lt());
                        if (mi < Lay::MC) {
                            mlist[mi] = e;
                        } else {
                            // the merge list is full: this lane merges the source itself
                            const unsigned long long v = slots[e & 0xffffu];
                            const uint32_t s = (uint32_t)(v >> 32), lo = (uint32_t)v;
                            const uint32_t c = lo & 0x3ffu, jm = lo >> 21, smx = (lo >> 10) & 0x7ffu;
                            const uint32_t ls = e >> 16;
                            const uint4 sm = __ldg(smin + ls);
                            const uint32_t* st = a.tok + fa.meta[s].x;
                            const uint32_t xq = qsrc[jm], qrest = lq - jm - 1;
                            const uint32_t k0 = smx != kSmaxUnknown ? smx + 1 : c;
                            uint32_t k = k0, cnt = c;
                            while (k < ls && cnt + min(ls - k, qrest - (cnt - c)) >= sm.y)
                                cnt += merge_step(st, k, ls, xq, bm, qmode, qsrc, lq);
                            ctr.merged += k - k0;
                            tally_overlap(a, ctr, q, s, cnt, sm.y, sm.z);
                        }
                    }
                }
            }
            my_cand = warp_sum(my_cand);
            if (lane == 0 && my_cand) atomicAdd(&s_cand, my_cand);
            __syncthreads();
            // 3. merge the listed sources (a warp per source) and clear the slots
            const uint32_t nm = min(s_nm, Lay::MC);
            for (uint32_t mi = wid; mi < nm; mi += NW) {
                const uint32_t e = mlist[mi];
                const unsigned long long v = slots[e & 0xffffu];
                const uint32_t s = (uint32_t)(v >> 32), lo = (uint32_t)v;
                const uint32_t c = lo & 0x3ffu, jm = lo >> 21, smx = (lo >> 10) & 0x7ffu;
                const uint32_t ls = e >> 16;
                const uint4 sm = __ldg(smin + ls);
                const uint32_t im = sm.y;
                const uint32_t* st = a.tok + fa.meta[s].x;
                const uint32_t xq = qsrc[jm], qrest = lq - jm - 1;
                const uint32_t k0 = smx != kSmaxUnknown ? smx + 1 : c;
                uint32_t k = k0, cnt = c;
                while (k < ls && cnt + min(ls - k, qrest - (cnt - c)) >= im) {
                    const uint32_t kk = k + lane;
                    bool hit = false;
                    if (kk < ls) {
                        const uint32_t x = __ldg(st + kk);
                        hit = x > xq && bm_test(bm, qmode, x, qsrc, 0, lq);
                    }
                    cnt += __popc(__ballot_sync(kFull, hit));
                    k = min(k + 32u, ls);
                }
                if (lane == 0) {
                    ctr.merged += k - k0;
                    tally_overlap(a, ctr, q, s, cnt, im, sm.z);
                }
            }
            __syncthreads();  // the merges read the slots
            // (the next barrier -- the next part's first, or the query's last -- orders
            // this clear before any later accumulate)
            for (uint32_t i2 = tid; i2 < nocc; i2 += NT) slots[occ[i2] & 0xffffu] = kEmptySlot;
            if (tid == 0) {
                s_nocc = 0;
                s_nm = 0;
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        ctr.cand += s_cand;
        ctr.window += s_win;
    }
    if (qmode == QM_HASH) {
        uint4* b4 = reinterpret_cast<uint4*>(bm);
        for (uint32_t i = tid; i < kQHashWords / 4; i += NT) b4[i] = make_uint4(0, 0, 0, 0);
    } else {
        for (uint32_t j = tid; j < lq; j += NT) {
            const uint32_t x = qsrc[j];
            const uint32_t b = qmode == QM_EXACT ? x : bloom_bit(x);
            bm[b >> 5] = 0u;
        }
    }
    __syncthreads();
}

// RT = resident threads per SM the register budget is sized for (launch
// bounds): 1024 caps a thread at 64 registers, 768 at 80, 512 at 128.
template <int NT, int HLOG, int RT, bool SIDED>
__global__ void __launch_bounds__(NT, RT / NT) k_fused(const JoinArgs* __restrict__ joins, const FusedArgs* __restrict__ fargs,
                                              const uint4* __restrict__ items, uint32_t n_items,
                                              uint32_t* item_counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    using Lay = FusedLayout<HLOG>;
    unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + Lay::off_bm);
    for (uint32_t h = threadIdx.x; h < Lay::H; h += NT) slots[h] = kEmptySlot;
    for (uint32_t i = threadIdx.x; i < Lay::BW; i += NT) bm[i] = 0u;
    __syncthreads();
    FusedCounters ctr = {0, 0, 0, 0, 0, 0, 0};
    // work items are claimed one ahead: thread 0 claims the next item as the
    // current one starts, so one barrier per item publishes it
    __shared__ uint32_t s_item[2];
    uint32_t cur_join = 0xffffffffu;
    if (threadIdx.x == 0) s_item[0] = atomicAdd(item_counter, 1u);
    __syncthreads();
    for (uint32_t r = 0;; r ^= 1u) {
        const uint32_t it = s_item[r];
        if (it >= n_items) break;
        if (threadIdx.x == 0) s_item[r ^ 1u] = atomicAdd(item_counter, 1u);
        const uint4 w = items[it];
        if (w.x != cur_join) {
            if (cur_join != 0xffffffffu) flush_fused_counters(joins[cur_join], ctr);
            cur_join = w.x;
        }
        const JoinArgs& a = joins[w.x];
        const FusedArgs& fa = fargs[w.x];
        for (uint32_t q = w.y; q < w.z; q++) fused_query<NT, HLOG, SIDED>(a, fa, q, smem, ctr);
        const uint32_t big = max(max(ctr.cand, ctr.window), max(ctr.merged, ctr.verified));
        if (__any_sync(kFull, big > (1u << 30))) flush_fused_counters(a, ctr);
        __syncthreads();
    }
    if (cur_join != 0xffffffffu) flush_fused_counters(joins[cur_join], ctr);
}

}  // namespace fgss
