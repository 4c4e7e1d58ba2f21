// join.cu -- host driver of the self-join stages (see join_kernels.cuh for
// the device side and the reference file:line of each stage).
#include <string.h>

#include <algorithm>

#include "join.h"
#include "prims.cuh"

namespace fgss {

namespace {

template <typename T>
void upload(Ctx& c, T* dst, const std::vector<T>& v) {
    FGSS_CK(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
}

__global__ void k_sum_u32(const uint32_t* __restrict__ in, uint64_t n, unsigned long long* out) {
    unsigned long long s = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += in[i];
    s = warp_sum(s);
    if (lane_id() == 0 && s) atomicAdd(out, s);
}

template <int MODE, int NT, int HLOG>
void set_smem_attr() {
    static bool done = false;
    if (!done) {
        FGSS_CK(cudaFuncSetAttribute(k_probe<MODE, NT, HLOG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ProbeLayout<MODE, HLOG>::bytes));
        done = true;
    }
}

}  // namespace

__global__ void k_widen(const uint32_t* in, uint64_t* out) { *out = *in; }

int bits_for(uint64_t v) {
    int b = 1;
    while (b < 64 && (1ull << b) < v) b++;
    return b;
}

DevBounds device_bounds(Ctx& c, float t, int mode) {
    uint32_t bits;
    memcpy(&bits, &t, 4);
    std::string k = "lut." + std::to_string(bits) + "." + std::to_string(mode) + ".";
    const size_t L = kMaxLen + 1, S = 2 * (size_t)kMaxLen + 1;
    bool fresh = c.bufs.find(k + "probe") == c.bufs.end();
    DevBounds d;
    d.probe = c.devT<uint16_t>(k + "probe", L);
    d.index = c.devT<uint16_t>(k + "index", L);
    d.minsz = c.devT<uint32_t>(k + "minsz", L);
    d.maxsz = c.devT<uint32_t>(k + "maxsz", L);
    d.lmin = c.devT<uint32_t>(k + "lmin", L);
    d.cand_min = c.devT<uint32_t>(k + "cand", S);
    d.inter_min = c.devT<uint32_t>(k + "inter", S);
    d.need = c.devT<uint32_t>(k + "need", S);
    d.smin = c.devT<uint4>(k + "smin", S);
    if (fresh) {
        BoundTables b;
        compute_bounds(t, mode, b);
        upload(c, d.probe, b.probe);
        upload(c, d.index, b.index);
        upload(c, d.minsz, b.minsz);
        upload(c, d.maxsz, b.maxsz);
        upload(c, d.lmin, b.lmin);
        upload(c, d.cand_min, b.cand_min);
        upload(c, d.inter_min, b.inter_min);
        upload(c, d.need, b.need);
        std::vector<uint4> sm(S);
        for (size_t i = 0; i < S; i++) sm[i] = make_uint4(b.cand_min[i], b.inter_min[i], b.need[i], 0u);
        upload(c, d.smin, sm);
        c.sync();  // the host vectors go out of scope
    }
    return d;
}

void join_setup_host(Ctx& c, JoinState& J, const fgss_sets_view& v, const fgss_join_opts& o, int slot) {
    J.slot = slot;
    J.t = o.threshold;
    J.res_cap_user = o.result_capacity;
    J.bounds = o.bounds;
    J.filter = o.filter;
    if (o.filter < FGSS_FILTER_AUTO || o.filter > FGSS_FILTER_GLOBAL) fail(FGSS_ERR_INVALID, "unknown filter strategy");
    if (!(o.threshold > 0.0f && o.threshold < 1.0f))
        fail(FGSS_ERR_INVALID, "threshold must be in (0, 1) (fgssjoin_cli.cu:31-35)");
    if (v.n_sets >= 0xffffffffull) fail(FGSS_ERR_UNSUPPORTED, "more than 2^32-1 records");
    if (v.n_tokens >= 0xffffffffull) fail(FGSS_ERR_UNSUPPORTED, "more than 2^32-1 tokens");
    const uint64_t n = v.n_sets, T = v.n_tokens;
    J.in = v;
    if (!v.on_device) {
        uint32_t* pos = c.devT<uint32_t>(J.pfx("in.pos"), n + 1);
        uint32_t* len = c.devT<uint32_t>(J.pfx("in.len"), n + 1);
        uint32_t* tok = c.devT<uint32_t>(J.pfx("in.tok"), T + 1);
        uint32_t* id = v.id ? c.devT<uint32_t>(J.pfx("in.id"), n + 1) : nullptr;
        if (n) {
            FGSS_CK(cudaMemcpyAsync(pos, v.pos, n * 4, cudaMemcpyHostToDevice, c.stream));
            FGSS_CK(cudaMemcpyAsync(len, v.len, n * 4, cudaMemcpyHostToDevice, c.stream));
            if (id) FGSS_CK(cudaMemcpyAsync(id, v.id, n * 4, cudaMemcpyHostToDevice, c.stream));
        }
        if (T) FGSS_CK(cudaMemcpyAsync(tok, v.tokens, T * 4, cudaMemcpyHostToDevice, c.stream));
        J.in.pos = pos;
        J.in.len = len;
        J.in.tokens = tok;
        J.in.id = id;
        J.in.on_device = 1;
    }
    J.id = J.in.id;
    J.lut = device_bounds(c, J.t, J.bounds);

    JoinArgs& a = J.args;
    memset(&a, 0, sizeof a);
    a.pos = J.in.pos;
    a.len = J.in.len;
    a.tok = J.in.tokens;
    a.n = (uint32_t)n;
    a.n_terms = v.n_terms;
    a.n_tokens = v.n_tokens;
    a.probe = J.lut.probe;
    a.index = J.lut.index;
    a.minsz = J.lut.minsz;
    a.maxsz = J.lut.maxsz;
    a.cand_min = J.lut.cand_min;
    a.inter_min = J.lut.inter_min;
    a.need = J.lut.need;
    a.lmin = J.lut.lmin;
    a.id = J.id;
    a.thr = J.t;
    a.side = J.side;
    a.heavy_cap = (uint32_t)n;
    a.join_id = (uint32_t)slot;
    a.heavy_min_qp = 0xffffffffu;  // set by the batched method's launch shape
    if (o.query_end > o.query_begin) {
        if (o.query_end > n) fail(FGSS_ERR_INVALID, "query_end beyond the number of records");
        a.q_lo = (uint32_t)o.query_begin;
        a.q_hi = (uint32_t)o.query_end;
    } else {
        a.q_lo = 0;
        a.q_hi = (uint32_t)n;
    }
    J.term_bits = bits_for((uint64_t)v.n_terms + 1);
}

void join_setup(Ctx& c, JoinState& J, const fgss_sets_view& v, const fgss_join_opts& o, int slot, bool check) {
    join_setup_host(c, J, v, o, slot);
    const uint64_t n = J.in.n_sets;
    J.status = c.devT<uint32_t>(J.pfx("status"), 8);
    J.stats = c.devT<unsigned long long>(J.pfx("stats"), SS_N);
    J.maxlen = J.status + 1;
    FGSS_CK(cudaMemsetAsync(J.status, 0, 32, c.stream));
    FGSS_CK(cudaMemsetAsync(J.stats, 0, SS_N * 8, c.stream));
    J.icnt = c.devT<uint32_t>(J.pfx("icnt"), n + 1);
    J.pcnt = c.devT<uint32_t>(J.pfx("pcnt"), n + 1);
    J.d_e = c.devT<uint64_t>(J.pfx("E"), 2);
    uint32_t* send = c.devT<uint32_t>(J.pfx("send"), kMaxLen + 1);
    JoinArgs& a = J.args;
    a.status = J.status;
    a.stats = J.stats;
    a.send = send;
    a.heavy_q = c.devT<uint32_t>(J.pfx("heavy_q"), n + 1);
    a.heavy_count = J.status + 2;
    if (n == 0) return;
    k_prep<<<grid_for(n, 256, c.num_sms * 16), 256, 0, c.stream>>>(a, J.icnt, J.pcnt, J.maxlen, 1);
    FGSS_LAUNCH_CK();
    k_send<<<grid_for(kMaxLen + 1, 256), 256, 0, c.stream>>>(J.in.len, (uint32_t)n, J.lut.lmin, send, kMaxLen + 1);
    FGSS_LAUNCH_CK();
    // no kernel reads tokens through caller offsets before they are validated
    uint32_t* h = c.pinnedT<uint32_t>(J.pfx("h.prep"), 4);
    FGSS_CK(cudaMemcpyAsync(h, J.status, 4, cudaMemcpyDeviceToHost, c.stream));
    if (!check) return;
    c.sync();
    join_check_input(c, J);
}

void join_check_input(Ctx& c, JoinState& J) {
    if (J.in.n_sets == 0) return;
    check_input_status(c.pinnedT<uint32_t>(J.pfx("h.prep"), 4)[0]);
}

void check_input_status(uint32_t st) {
    if (st & ST_BAD_OFFSETS) fail(FGSS_ERR_FORMAT, "a record's pos + len exceeds n_tokens");
    if (st & ST_TOO_LONG) fail(FGSS_ERR_UNSUPPORTED, "a record has more than 65535 tokens");
    if (st & ST_BAD_TOKENS)
        fail(FGSS_ERR_FORMAT, "tokens must be strictly ascending inside each record and below n_terms");
}

void join_index(Ctx& c, JoinState& J) {
    const uint64_t n = J.in.n_sets, T = J.in.n_tokens;
    JoinArgs& a = J.args;
    uint32_t* ioff = c.devT<uint32_t>(J.pfx("ioff"), n + 1);
    uint32_t* e32 = c.devT<uint32_t>(J.pfx("E32"), 2);
    uint32_t* list_off = c.devT<uint32_t>(J.pfx("list_off"), (uint64_t)J.in.n_terms + 2);
    uint2* ent = c.devT<uint2>(J.pfx("ent"), T + 1);
    a.list_off = list_off;
    a.ent = ent;
    if (n == 0) {
        FGSS_CK(cudaMemsetAsync(list_off, 0, ((uint64_t)J.in.n_terms + 1) * 4, c.stream));
        FGSS_CK(cudaMemsetAsync(J.d_e, 0, 8, c.stream));
        return;
    }
    exclusive_scan<uint32_t>(c, J.icnt, ioff, n, nullptr, e32, J.pfx("scan.i").c_str());
    k_widen<<<1, 1, 0, c.stream>>>(e32, J.d_e);
    FGSS_LAUNCH_CK();
    // entries: capacity T (index prefix <= record length); count from the device
    uint32_t* key = c.devT<uint32_t>(J.pfx("ix.key"), T + 1);
    uint64_t* val = c.devT<uint64_t>(J.pfx("ix.val"), T + 1);
    k_index_entries<<<grid_for(n * 32, 256, c.num_sms * 32), 256, 0, c.stream>>>(a, ioff, key, val);
    FGSS_LAUNCH_CK();
    radix_sort<uint32_t, uint64_t>(c, key, val, T, J.d_e, 0, J.term_bits, J.pfx("ixsort").c_str());
    k_index_lists<<<grid_for(T, 256, c.num_sms * 32), 256, 0, c.stream>>>(key, val, J.d_e, J.in.n_terms, list_off,
                                                                         ent);
    FGSS_LAUNCH_CK();
}

void join_finish_status(Ctx& c, JoinState& J) {
    uint32_t* h = c.pinnedT<uint32_t>(J.pfx("h.status"), 4);
    unsigned long long* hs = c.pinnedT<unsigned long long>(J.pfx("h.stats"), SS_N);
    FGSS_CK(cudaMemcpyAsync(h, J.status, 16, cudaMemcpyDeviceToHost, c.stream));
    FGSS_CK(cudaMemcpyAsync(hs, J.stats, SS_N * 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    apply_status(J, h[0], hs);
}

void apply_status(JoinState& J, uint32_t st, const unsigned long long* stats) {
    J.status_host = st;
    memcpy(J.stats_host, stats, sizeof(J.stats_host));
    if (J.status_host & ST_TOO_LONG) fail(FGSS_ERR_UNSUPPORTED, "a record has more than 65535 tokens");
    if (J.status_host & ST_BAD_TOKENS)
        fail(FGSS_ERR_FORMAT, "tokens must be strictly ascending inside each record and below n_terms");
    if (J.status_host & (ST_HASH_FULL | ST_HEAVY_OVERFLOW))
        fail(FGSS_ERR_CUDA, "internal table overflow in the filter (status " + std::to_string(J.status_host) + ")");
}

HeavyScratch heavy_scratch(Ctx& c, const std::string& prefix, uint64_t n, uint32_t slots, bool capture) {
    HeavyScratch h;
    h.zero_words = (2 * n + 63) & ~63ull;
    h.aux_words = (2 * n + 65536 + 65537 + 63) & ~63ull;
    const std::string zn = prefix + "heavy.zero";
    auto it = c.bufs.find(zn);
    const size_t need = h.zero_words * slots * 4;
    const bool grow = it == c.bufs.end() || it->second.bytes < need;
    if (grow && capture) fail(FGSS_ERR_CUDA, "heavy scratch would grow inside a graph capture");
    h.zero = (uint32_t*)c.dev(zn, need);
    if (grow) FGSS_CK(cudaMemsetAsync(h.zero, 0, c.bufs[zn].bytes, c.stream));
    h.aux = c.devT<uint32_t>(prefix + "heavy.aux", h.aux_words * slots);
    return h;
}

void join_plain_filter_verify(Ctx& c, JoinState& J, bool want_cand) {
    const uint64_t n = J.in.n_sets;
    JoinArgs& a = J.args;
    constexpr int NT = 256, HL = 12;
    a.vcnt = c.devT<uint32_t>(J.pfx("vcnt"), n + 1);
    a.ccnt = c.devT<uint32_t>(J.pfx("ccnt"), n + 1);
    a.wcnt = c.devT<uint32_t>(J.pfx("wcnt"), n + 1);
    uint32_t* voff = c.devT<uint32_t>(J.pfx("voff"), n + 1);
    a.voff = voff;
    J.d_args = c.devT<JoinArgs>(J.pfx("args"), 1);
    uint32_t* hcnt = c.pinnedT<uint32_t>(J.pfx("h.cnt"), 8);
    uint32_t* tot = c.devT<uint32_t>(J.pfx("tot"), 8);
    uint32_t* qctr = c.devT<uint32_t>(J.pfx("qctr"), 2);
    if (n == 0) {
        J.n_res = 0;
        return;
    }
    FGSS_CK(cudaMemsetAsync(a.vcnt, 0, n * 4, c.stream));
    FGSS_CK(cudaMemsetAsync(a.ccnt, 0, n * 4, c.stream));
    FGSS_CK(cudaMemsetAsync(a.wcnt, 0, n * 4, c.stream));
    // ---- count pass
    FGSS_CK(cudaMemsetAsync(a.heavy_count, 0, 4, c.stream));
    FGSS_CK(cudaMemcpyAsync(J.d_args, &a, sizeof a, cudaMemcpyHostToDevice, c.stream));
    set_smem_attr<MODE_COUNT, NT, HL>();
    k_probe<MODE_COUNT, NT, HL><<<(unsigned)n, NT, ProbeLayout<MODE_COUNT, HL>::bytes, c.stream>>>(J.d_args, nullptr,
                                                                                                   0, nullptr);
    FGSS_LAUNCH_CK();
    FGSS_CK(cudaMemcpyAsync(hcnt, a.heavy_count, 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    const uint32_t nheavy = hcnt[0];
    HeavyScratch hs;
    uint32_t hslots = std::min<uint32_t>(nheavy, (uint32_t)c.num_sms);
    if (nheavy) {
        hs = heavy_scratch(c, "", n, hslots, false);
        FGSS_CK(cudaMemsetAsync(qctr, 0, 4, c.stream));
        k_probe_heavy<MODE_COUNT, 512><<<hslots, 512, 0, c.stream>>>(J.d_args, 0, 1, hs.zero, hs.zero_words, hs.aux,
                                                                     hs.aux_words, qctr);
        FGSS_LAUNCH_CK();
    }
    exclusive_scan<uint32_t>(c, a.vcnt, voff, n, nullptr, tot, J.pfx("scan.v").c_str());
    // logged per-query counters -> the reference's totals
    k_sum_u32<<<grid_for(n, 256, c.num_sms * 8), 256, 0, c.stream>>>(a.ccnt, n, &J.stats[SS_CANDIDATES]);
    FGSS_LAUNCH_CK();
    k_sum_u32<<<grid_for(n, 256, c.num_sms * 8), 256, 0, c.stream>>>(a.wcnt, n, &J.stats[SS_WINDOW]);
    FGSS_LAUNCH_CK();
    FGSS_CK(cudaMemcpyAsync(hcnt, tot, 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    const uint64_t C = hcnt[0];
    // ---- fill pass
    uint4* cand = c.devT<uint4>(J.pfx("cand"), C + 1);
    a.cand = cand;
    FGSS_CK(cudaMemsetAsync(a.heavy_count, 0, 4, c.stream));
    FGSS_CK(cudaMemcpyAsync(J.d_args, &a, sizeof a, cudaMemcpyHostToDevice, c.stream));
    set_smem_attr<MODE_FILL, NT, HL>();
    k_probe<MODE_FILL, NT, HL><<<(unsigned)n, NT, ProbeLayout<MODE_FILL, HL>::bytes, c.stream>>>(J.d_args, nullptr, 0,
                                                                                                 nullptr);
    FGSS_LAUNCH_CK();
    if (nheavy) {
        FGSS_CK(cudaMemsetAsync(qctr, 0, 4, c.stream));
        k_probe_heavy<MODE_FILL, 512><<<hslots, 512, 0, c.stream>>>(J.d_args, 0, 1, hs.zero, hs.zero_words, hs.aux,
                                                                    hs.aux_words, qctr);
        FGSS_LAUNCH_CK();
    }
    uint64_t* d_nc = c.devT<uint64_t>(J.pfx("nc"), 2);
    FGSS_CK(cudaMemcpyAsync(d_nc, &C, 8, cudaMemcpyHostToDevice, c.stream));
    if (want_cand) {
        std::vector<uint4> hc(C);
        if (C) FGSS_CK(cudaMemcpyAsync(hc.data(), cand, C * 16, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        J.cand_host.resize(3 * C);
        for (uint64_t i = 0; i < C; i++) {
            J.cand_host[3 * i] = hc[i].x;
            J.cand_host[3 * i + 1] = hc[i].y;
            J.cand_host[3 * i + 2] = hc[i].z;
        }
    }
    // ---- verification (thread-per-candidate merge in the reference; warp per candidate here)
    uint32_t* ov = c.devT<uint32_t>(J.pfx("ov"), C + 1);
    if (C) {
        // token bitmaps of every record (the same filter the batched method uses)
        const uint32_t bmw = bitmap_words(J.in.n_tokens, n);
        uint4* bmap = c.devT<uint4>(J.pfx("bmap"), (uint64_t)bmw * n + 4);
        k_bitmaps<<<grid_for(n * 32, 256, c.num_sms * 64), 256, 0, c.stream>>>(a, bmap, bmw);
        FGSS_LAUNCH_CK();
        k_verify<<<grid_for(C * 32, 256, c.num_sms * 64), 256, 0, c.stream>>>(a, cand, d_nc, ov, bmap, bmw);
        FGSS_LAUNCH_CK();
    }
    // ---- compaction of the verified pairs: count -> scan -> fill
    uint32_t* flag = c.devT<uint32_t>(J.pfx("flag"), C + 1);
    uint32_t* off = c.devT<uint32_t>(J.pfx("off"), C + 1);
    uint64_t R = 0;
    if (C) {
        k_result_flags<<<grid_for(C, 256, c.num_sms * 32), 256, 0, c.stream>>>(a, cand, ov, d_nc, flag);
        FGSS_LAUNCH_CK();
        exclusive_scan<uint32_t>(c, flag, off, C, nullptr, tot + 2, J.pfx("scan.r").c_str());
        FGSS_CK(cudaMemcpyAsync(hcnt + 2, tot + 2, 4, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        R = hcnt[2];
    }
    uint64_t* keys = c.devT<uint64_t>(J.pfx("rkey"), R + 1);
    uint32_t* vals = c.devT<uint32_t>(J.pfx("rval"), R + 1);
    if (R) {
        k_result_fill<<<grid_for(C, 256, c.num_sms * 32), 256, 0, c.stream>>>(cand, ov, flag, off, d_nc, keys, vals);
        FGSS_LAUNCH_CK();
    }
    J.d_nres = c.devT<uint64_t>(J.pfx("nres"), 2);
    FGSS_CK(cudaMemcpyAsync(J.d_nres, &R, 8, cudaMemcpyHostToDevice, c.stream));
    join_output(c, J, keys, vals, J.d_nres, R);
    J.n_res = R;
    c.sync();
}

void join_output(Ctx& c, JoinState& J, uint64_t* keys, uint32_t* vals, const uint64_t* d_n, uint64_t n_cap) {
    const uint64_t n = J.in.n_sets;
    J.oq = c.devT<uint32_t>(J.pfx("o.q"), n_cap + 1);
    J.os = c.devT<uint32_t>(J.pfx("o.s"), n_cap + 1);
    J.oidq = c.devT<uint32_t>(J.pfx("o.idq"), n_cap + 1);
    J.oids = c.devT<uint32_t>(J.pfx("o.ids"), n_cap + 1);
    J.oo = c.devT<uint32_t>(J.pfx("o.o"), n_cap + 1);
    J.osim = c.devT<float>(J.pfx("o.sim"), n_cap + 1);
    if (n_cap == 0) return;
    // keys are (q << 32 | s); the sort only needs the bits that vary
    int b = bits_for(n);
    radix_sort<uint64_t, uint32_t>(c, keys, vals, n_cap, d_n, 0, b, J.pfx("rsort.lo").c_str());
    radix_sort<uint64_t, uint32_t>(c, keys, vals, n_cap, d_n, 32, 32 + b, J.pfx("rsort.hi").c_str());
    k_result_out<<<grid_for(n_cap, 256, c.num_sms * 32), 256, 0, c.stream>>>(keys, vals, d_n, J.id, J.in.len, J.oq,
                                                                             J.os, J.oidq, J.oids, J.oo, J.osim);
    FGSS_LAUNCH_CK();
}

}  // namespace fgss
