// batch_kernels.cuh -- the batched method's per-record stages for every join
// of a batch in one launch each (the tile table: tiles.cuh).  The joins'
// per-record arrays are slices of batch-level buffers; the bodies are the
// per-join stages' own (join_kernels.cuh, fused_kernels.cuh).
#pragma once

#include "fused_kernels.cuh"
#include "tiles.cuh"

namespace fgss {

// k_prep for every join: counts into the batch arrays icnt / pcnt (record g).
static __global__ void k_prep_mj(const JoinArgs* __restrict__ joins, TileMap m, uint32_t* __restrict__ icnt,
                                 uint32_t* __restrict__ pcnt) {
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange t = tile_range(m, b);
        const JoinArgs& a = joins[t.j];
        const uint64_t g0 = __ldg(m.roff + t.j);
        uint32_t local_max = 0, bad = 0;
        unsigned long long probe = 0;
        for (uint32_t i = t.r0 + threadIdx.x; i < t.r1; i += blockDim.x)
            prep_record(a, i, icnt + g0 + i, pcnt + g0 + i, local_max, bad, probe, 1);
        prep_flush(a, a.status + 1, local_max, bad, probe);
        if (t.r0 == 0 && threadIdx.x == 0) prep_skip_test(a);
    }
}

// send[L] of every join for the query lengths L <= its longest record (the
// only ones read); launched over nj x 65536 lengths.
static __global__ void k_send_mj(const JoinArgs* __restrict__ joins, uint32_t nj, uint32_t* __restrict__ send_all) {
    const uint64_t total = (uint64_t)nj << 16;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(x >> 16), L = (uint32_t)(x & 0xffffu);
        const JoinArgs& a = joins[j];
        if (L > a.status[1]) continue;  // longer than every record of the join
        send_all[(uint64_t)j * 65537 + L] = send_of(a.len, a.n, a.lmin[L]);
    }
}

// Index entries of every join (warp per record) with keys join << tbits | term
// (K: 32-bit keys when join and term bits fit).
template <typename K>
__global__ void k_index_entries_mj(const JoinArgs* __restrict__ joins, TileMap m, const uint32_t* __restrict__ ioff,
                                   uint32_t tbits, K* __restrict__ key, uint64_t* __restrict__ val) {
    const uint32_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange t = tile_range(m, b);
        const uint64_t g0 = __ldg(m.roff + t.j);
        for (uint32_t i = t.r0 + wid; i < t.r1; i += nw)
            index_entries_record<K>(joins[t.j], i, ioff[g0 + i], (K)t.j << tbits, key, val);
    }
}

// After the stable sort by (join, term): the entry columns and every join's
// list offsets, as positions in the batch's entry arrays (a join without
// entries keeps the zero offsets its buffer was cleared to).
template <typename K>
__global__ void k_index_lists_mj(const JoinArgs* __restrict__ joins, const K* __restrict__ key,
                                        const uint64_t* __restrict__ val, const uint64_t* __restrict__ d_e,
                                        uint32_t tbits, const uint64_t* __restrict__ loff,
                                        uint32_t* __restrict__ list_all, uint2* __restrict__ ent) {
    const uint64_t E = *d_e;
    const uint64_t tmask = (1ull << tbits) - 1;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < E; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = val[k], kk = (uint64_t)key[k];
        ent[k] = make_uint2((uint32_t)(v >> 32), (uint32_t)v);
        const uint32_t j = (uint32_t)(kk >> tbits), w = (uint32_t)(kk & tmask);
        uint32_t* lo = list_all + loff[j];
        if (k == 0 || (uint32_t)((uint64_t)key[k - 1] >> tbits) != j)
            for (uint32_t x = 0; x <= w; x++) lo[x] = (uint32_t)k;  // terms before the join's first
        uint32_t nxt = joins[j].n_terms;
        if (k + 1 < E && (uint32_t)((uint64_t)key[k + 1] >> tbits) == j) nxt = (uint32_t)((uint64_t)key[k + 1] & tmask);
        for (uint32_t x = w + 1; x <= nxt; x++) lo[x] = (uint32_t)(k + 1);
    }
}

// Number of index entries of every join (from the batch's entry offsets).
static __global__ void k_join_entries(const uint64_t* __restrict__ roff, uint32_t nj,
                                      const uint32_t* __restrict__ ioff, uint64_t* __restrict__ d_e_all) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x)
        d_e_all[2 * j] = (uint64_t)(ioff[roff[j + 1]] - ioff[roff[j]]);
}

// Warp per record: the windows of every probe token (windows_query) of every join.
static __global__ void k_windows_mj(const JoinArgs* __restrict__ joins, TileMap m, const uint32_t* __restrict__ poff,
                                    uint2* __restrict__ win, uint32_t* __restrict__ wpre, uint32_t* __restrict__ wtot,
                                    uint4* __restrict__ meta) {
    const uint32_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange t = tile_range(m, b);
        const uint64_t g0 = __ldg(m.roff + t.j);
        for (uint32_t q = t.r0 + wid; q < t.r1; q += nw)
            windows_query(joins[t.j], q, poff + g0, win, wpre, wtot + g0, meta + g0);
    }
}

// Warp per record: every join's token bitmaps.
static __global__ void k_bitmaps_mj(const JoinArgs* __restrict__ joins, const FusedArgs* __restrict__ fargs,
                                    TileMap m) {
    __shared__ uint32_t sw[8][16];  // launched with 256 threads: a bitmap per warp
    const uint32_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange t = tile_range(m, b);
        const FusedArgs& fa = fargs[t.j];
        uint4* bmap = const_cast<uint4*>(fa.bmap);
        for (uint32_t r = t.r0 + wid; r < t.r1; r += nw) bitmap_record(joins[t.j], r, bmap, fa.bmw, sw[wid]);
    }
}

// Warp per record: every join's chunk splits (chunks_query), one boundary buffer.
static __global__ void k_chunks_mj(const JoinArgs* __restrict__ joins, const FusedArgs* __restrict__ fargs, TileMap m,
                                   const uint32_t* __restrict__ wtot, uint32_t cap, uint32_t* __restrict__ cbuf,
                                   uint64_t cbuf_cap, unsigned long long* __restrict__ cbuf_used) {
    const uint32_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange t = tile_range(m, b);
        const FusedArgs& fa = fargs[t.j];
        const uint64_t g0 = __ldg(m.roff + t.j);
        for (uint32_t q = t.r0 + wid; q < t.r1; q += nw)
            chunks_query(joins[t.j], q, fa.poff, fa.win, wtot + g0, cap, const_cast<uint2*>(fa.qchunk), cbuf,
                         cbuf_cap, cbuf_used);
    }
}

// Features of the learned cost model for query q (warp-collective; lane 0
// writes the kFeatures floats to f): log sizes of the query, its probe
// prefix, the summed and longest full lists of its probe tokens, their mean
// log length, its id window, its position and the threshold.
constexpr int kFeatures = 8;
__device__ __forceinline__ void features_record(const JoinArgs& a, uint32_t q, float* __restrict__ f) {
    const uint32_t lane = lane_id();
    const uint32_t lq = a.len[q];
    const uint32_t qp = lq <= 65535u ? a.probe[lq] : 0;
    const uint32_t* qt = a.tok + a.pos[q];
    unsigned long long sum = 0;
    uint32_t mx = 0;
    float slog = 0.f;
    for (uint32_t j = lane; j < qp; j += 32) {
        const uint32_t w = __ldg(qt + j);
        const uint32_t l = __ldg(a.list_off + w + 1) - __ldg(a.list_off + w);
        sum += l;
        mx = max(mx, l);
        slog += log1pf((float)l);
    }
    sum = warp_sum(sum);
    mx = __reduce_max_sync(kFull, mx);
    slog = warp_sum(slog);
    if (lane == 0) {
        const uint32_t send = lq <= 65535u ? a.send[lq] : q + 1;
        const uint32_t win = send > q + 1 ? send - q - 1 : 0;
        f[0] = log1pf((float)lq);
        f[1] = log1pf((float)qp);
        f[2] = log1pf((float)sum);
        f[3] = log1pf((float)mx);
        f[4] = qp ? slog / (float)qp : 0.f;
        f[5] = log1pf((float)win);
        f[6] = a.n ? (float)q / (float)a.n : 0.f;
        f[7] = a.thr;
    }
}

// Warp per record: every join's features, at the record's batch index.
static __global__ void k_features_mj(const JoinArgs* __restrict__ joins, TileMap m, float* __restrict__ feat) {
    const uint32_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange tr = tile_range(m, b);
        const uint64_t g0 = __ldg(m.roff + tr.j);
        for (uint32_t q = tr.r0 + wid; q < tr.r1; q += nw) features_record(joins[tr.j], q, feat + (g0 + q) * kFeatures);
    }
}

// Work-item cost of every query: exact window entries + 4 x the learned
// estimate of its candidates (when given) + its size; 0 outside the join's
// query range.  Also sums into *need the chunk-boundary words the queries'
// splits for slot tables of `cap` entries take (chunks_query).
static __global__ void k_cost_mj(const JoinArgs* __restrict__ joins, TileMap m, const uint32_t* __restrict__ wtot,
                                 const uint32_t* __restrict__ pred, uint32_t cap, uint64_t* __restrict__ cost,
                                 unsigned long long* __restrict__ need) {
    unsigned long long words = 0;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange tr = tile_range(m, b);
        const JoinArgs& a = joins[tr.j];
        const uint64_t g0 = __ldg(m.roff + tr.j);
        for (uint32_t q = tr.r0 + threadIdx.x; q < tr.r1; q += blockDim.x) {
            unsigned long long v = 0;
            const uint32_t L = wtot[g0 + q];
            if (q >= a.q_lo && q < a.q_hi) {
                v = (unsigned long long)L + a.len[q];
                if (pred) v += 4ull * pred[g0 + q];
            }
            cost[g0 + q] = v;
            uint32_t qp, span;
            words += (unsigned long long)(chunk_count(a, q, L, cap, qp, span) - 1) * qp;
        }
    }
    words = warp_sum(words);
    if (lane_id() == 0 && words) atomicAdd(need, words);
}

// Cost total of every join from the batch's exclusive cost prefix.
static __global__ void k_join_cost_totals(const uint64_t* __restrict__ roff, uint32_t nj,
                                          const uint64_t* __restrict__ cpre, uint64_t* __restrict__ tot) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x)
        tot[j] = cpre[roff[j + 1]] - cpre[roff[j]];
}

// The join of batch-wide item k: the last j with koff[j] <= k.
__device__ __forceinline__ uint32_t item_join(const uint32_t* __restrict__ koff, uint32_t nj, uint32_t k) {
    uint32_t lo = 0, hi = nj;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (koff[mid + 1] <= k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Work items of every join: item k of join j (K = koff[j+1] - koff[j] items) =
// its queries with cost prefix in [k * target, (k+1) * target), and its sort
// key: the cost as a float's exponent and top 7 mantissa bits, complemented so
// an ascending sort puts the costliest first (16 bits, two radix passes).
static __global__ void k_items_mj(const uint64_t* __restrict__ roff, const uint32_t* __restrict__ koff, uint32_t nj,
                                  uint32_t nitems, const uint64_t* __restrict__ cpre, const uint64_t* __restrict__ tot,
                                  uint4* __restrict__ items, uint32_t* __restrict__ key, uint32_t* __restrict__ val) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < nitems; x += gridDim.x * blockDim.x) {
        const uint32_t j = item_join(koff, nj, x);
        const uint32_t K = koff[j + 1] - koff[j], k = x - koff[j];
        const uint64_t g0 = roff[j];
        const uint32_t n = (uint32_t)(roff[j + 1] - g0);
        const uint64_t base = cpre[g0], total = tot[j];
        const uint64_t target = (total + K - 1) / K;
        auto first_ge = [&](uint64_t y) {  // first local q with cost prefix >= y
            uint32_t lo = 0, hi = n;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (cpre[g0 + mid] - base < y) lo = mid + 1;
                else hi = mid;
            }
            return lo;
        };
        const uint32_t qb = k == 0 ? 0 : first_ge(k * target);
        const uint32_t qe = k + 1 == K ? n : first_ge((k + 1) * target);
        const uint32_t e = max(qb, qe);
        items[x] = make_uint4(j, qb, e, 0);
        const uint64_t cb = qb < n ? cpre[g0 + qb] - base : total, ce = e < n ? cpre[g0 + e] - base : total;
        key[x] = (~__float_as_uint((float)(ce - cb)) >> 16) & 0xffffu;
        val[x] = x;
    }
}

// Resets every join's filter counters and overflow bits before a re-run (the
// input-validation bits and the probe-token count stay).
static __global__ void k_clear_filter_state_mj(const JoinArgs* __restrict__ joins, uint32_t nj) {
    for (uint32_t j = blockIdx.x; j < nj; j += gridDim.x) {
        const JoinArgs& a = joins[j];
        if (threadIdx.x == 0) {
            a.status[0] &= ~(uint32_t)(ST_RES_OVERFLOW | ST_HEAVY_OVERFLOW | ST_HASH_FULL);
            a.status[2] = 0;
            a.status[3] = 0;
        }
        if (threadIdx.x < SS_N && threadIdx.x != SS_PROBE) a.stats[threadIdx.x] = 0;
    }
}

// One CTA: every join's result count (at most its capacity), their exclusive
// prefix resoff[0..nj] and the total *d_n.
static __global__ void k_result_offsets(const JoinArgs* __restrict__ joins, uint32_t nj, uint64_t* __restrict__ resoff,
                                        uint64_t* __restrict__ d_n) {
    __shared__ unsigned long long wsum[33];
    unsigned long long carry = 0;
    for (uint32_t b = 0; b < nj; b += blockDim.x) {
        const uint32_t j = b + threadIdx.x;
        unsigned long long c = 0;
        if (j < nj) c = min(*joins[j].res_count, joins[j].res_cap);
        unsigned long long tot;
        const unsigned long long pre = block_excl_scan<unsigned long long>(c, wsum, &tot);
        if (j < nj) resoff[j] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        resoff[nj] = carry;
        *d_n = carry;
    }
}

// Every join's results as sort keys join << 2 qb | q << qb | s (value: the
// overlap), packed at resoff[j]; tiles over the result capacities.
static __global__ void k_result_keys_mj(const JoinArgs* __restrict__ joins, TileMap m, const uint64_t* __restrict__ resoff,
                                        uint32_t qb, uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange tr = tile_range(m, b);
        const JoinArgs& a = joins[tr.j];
        const uint32_t cnt = min(*a.res_count, a.res_cap);
        const uint64_t o = resoff[tr.j];
        const uint64_t tag = (uint64_t)tr.j << (2 * qb);
        for (uint32_t i = tr.r0 + threadIdx.x; i < min(tr.r1, cnt); i += blockDim.x) {
            key[o + i] = tag | ((uint64_t)a.res_q[i] << qb) | a.res_s[i];
            val[o + i] = a.res_o[i];
        }
    }
}

// Sorted keys -> every join's output columns (q, s, id_q, id_s, overlap, sim),
// join j's at capoff[j] in the batch's output arrays.
static __global__ void k_result_out_mj(const JoinArgs* __restrict__ joins, const uint64_t* __restrict__ key,
                                       const uint32_t* __restrict__ val, const uint64_t* __restrict__ d_n,
                                       const uint64_t* __restrict__ resoff, const uint64_t* __restrict__ capoff,
                                       uint32_t qb, uint32_t* __restrict__ oq, uint32_t* __restrict__ os,
                                       uint32_t* __restrict__ oidq, uint32_t* __restrict__ oids,
                                       uint32_t* __restrict__ oo, float* __restrict__ osim) {
    const uint64_t n = *d_n;
    const uint64_t qmask = (1ull << qb) - 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[i];
        const uint32_t j = (uint32_t)(k >> (2 * qb));
        const uint32_t q = (uint32_t)((k >> qb) & qmask), s = (uint32_t)(k & qmask), o = val[i];
        const JoinArgs& a = joins[j];
        const uint64_t d = capoff[j] + (i - resoff[j]);
        oq[d] = q;
        os[d] = s;
        oidq[d] = a.id ? a.id[q] : q;
        oids[d] = a.id ? a.id[s] : s;
        oo[d] = o;
        const uint32_t uni = a.len[q] + a.len[s] - o;
        osim[d] = __fdiv_rn(__uint2float_rn(o), __uint2float_rn(uni));  // similarity.cuh:78-82
    }
}

}  // namespace fgss
