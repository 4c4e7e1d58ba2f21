// rsjoin.cu -- the R-S join: pairs (r, s) with r a record of R, s a record of
// S (one shared vocabulary) and Jaccard >= t.
//
// The reference has no R-S join: its preprocess CLI names a "dualjoin" mode
// (src/preprocess_cli.cpp:22-32,93-119) that reads only its first file.  The
// join here is defined as the self-join of R and S together restricted to the
// pairs across: the union is put in memory order (descending size, R before S
// at equal size, then the index within its side), every self-join stage runs
// on it unchanged, and a one-byte side per record makes the filters skip
// entries of the query's own side before anything else, so the candidate and
// result counters count cross pairs only.  The pairs are then mapped back to
// (index in R, index in S) and sorted by that.  With FGSS_BOUNDS_EXACT the
// result is exactly the set of pairs with J >= t; with the reference's float32
// bounds it has the self-join's boundary behaviour.
#include <string.h>

#include "join.h"
#include "prims.cuh"

namespace fgss {

namespace {

int bits_needed(uint64_t v) {  // bits to hold values < v
    int b = 1;
    while (b < 64 && (1ull << b) < v) b++;
    return b;
}

// Union sort keys: (0xffff - min(len, 0xffff)) << 32 | side << 31 | index.
__global__ void k_rs_keys(const uint32_t* __restrict__ rlen, uint32_t nr, const uint32_t* __restrict__ slen,
                          uint32_t ns, uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    const uint32_t n = nr + ns;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t side = i >= nr, idx = side ? i - nr : i;
        const uint32_t len = side ? slen[idx] : rlen[idx];
        key[i] = ((uint64_t)(0xffffu - min(len, 0xffffu)) << 32) | ((uint64_t)side << 31) | idx;
        val[i] = i;
    }
}

// Sorted keys -> union pos / len / side / index within the side.  A record
// whose pos + len leaves its own side's tokens sets bit 0 of *bad.
__global__ void k_rs_union(const uint64_t* __restrict__ key, uint32_t n, const uint32_t* __restrict__ rpos,
                           const uint32_t* __restrict__ rlen, uint64_t tr, const uint32_t* __restrict__ spos,
                           const uint32_t* __restrict__ slen, uint64_t ts, uint32_t* __restrict__ upos,
                           uint32_t* __restrict__ ulen, uint8_t* __restrict__ side, uint32_t* __restrict__ orig,
                           uint32_t* __restrict__ bad) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint64_t x = key[k];
        const uint32_t sd = (uint32_t)(x >> 31) & 1u, idx = (uint32_t)x & 0x7fffffffu;
        const uint32_t p = sd ? spos[idx] : rpos[idx];
        const uint32_t l = sd ? slen[idx] : rlen[idx];
        if ((uint64_t)p + l > (sd ? ts : tr)) atomicOr(bad, 1u);
        upos[k] = sd ? (uint32_t)(p + tr) : p;
        ulen[k] = l;
        side[k] = (uint8_t)sd;
        orig[k] = idx;
    }
}

// Union-index pairs (sorted by (q, s)) -> keys r << 32 | s in the sides' own
// indices, value = the pair's position.
__global__ void k_rs_remap(const uint32_t* __restrict__ oq, const uint32_t* __restrict__ os, uint64_t n,
                           const uint8_t* __restrict__ side, const uint32_t* __restrict__ orig,
                           uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = oq[i], b = os[i];
        const bool a_is_r = side[a] == 0;
        const uint32_t r = orig[a_is_r ? a : b], s = orig[a_is_r ? b : a];
        key[i] = ((uint64_t)r << 32) | s;
        val[i] = (uint32_t)i;
    }
}

__global__ void k_rs_out(const uint64_t* __restrict__ key, const uint32_t* __restrict__ val, uint64_t n,
                         const uint32_t* __restrict__ rid, const uint32_t* __restrict__ sid,
                         const uint32_t* __restrict__ oo, const float* __restrict__ osim, uint32_t* __restrict__ q,
                         uint32_t* __restrict__ s, uint32_t* __restrict__ idq, uint32_t* __restrict__ ids,
                         uint32_t* __restrict__ o, float* __restrict__ sim) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[i];
        const uint32_t r = (uint32_t)(k >> 32), x = (uint32_t)k, v = val[i];
        q[i] = r;
        s[i] = x;
        idq[i] = rid ? rid[r] : r;
        ids[i] = sid ? sid[x] : x;
        o[i] = oo[v];
        sim[i] = osim[v];
    }
}

// A side's arrays on the device (copied when the caller's are host memory).
fgss_sets_view rs_side_on_device(Ctx& c, const fgss_sets_view& v, const char* tag) {
    if (v.on_device) return v;
    fgss_sets_view d = v;
    const std::string t(tag);
    uint32_t* pos = c.devT<uint32_t>("rs." + t + ".pos", v.n_sets + 1);
    uint32_t* len = c.devT<uint32_t>("rs." + t + ".len", v.n_sets + 1);
    uint32_t* tok = c.devT<uint32_t>("rs." + t + ".tok", v.n_tokens + 1);
    uint32_t* id = v.id ? c.devT<uint32_t>("rs." + t + ".id", v.n_sets + 1) : nullptr;
    if (v.n_sets) {
        if (!v.pos || !v.len) fail(FGSS_ERR_INVALID, "null record arrays");
        FGSS_CK(cudaMemcpyAsync(pos, v.pos, v.n_sets * 4, cudaMemcpyHostToDevice, c.stream));
        FGSS_CK(cudaMemcpyAsync(len, v.len, v.n_sets * 4, cudaMemcpyHostToDevice, c.stream));
        if (id) FGSS_CK(cudaMemcpyAsync(id, v.id, v.n_sets * 4, cudaMemcpyHostToDevice, c.stream));
    }
    if (v.n_tokens) {
        if (!v.tokens) fail(FGSS_ERR_INVALID, "null token array");
        FGSS_CK(cudaMemcpyAsync(tok, v.tokens, v.n_tokens * 4, cudaMemcpyHostToDevice, c.stream));
    }
    d.pos = pos;
    d.len = len;
    d.tokens = tok;
    d.id = id;
    d.on_device = 1;
    return d;
}

}  // namespace

RsInput rs_union(Ctx& c, const fgss_sets_view& r_in, const fgss_sets_view& s_in) {
    if (r_in.n_sets >= 0x80000000ull || s_in.n_sets >= 0x80000000ull)
        fail(FGSS_ERR_UNSUPPORTED, "R-S join: more than 2^31-1 records on one side");
    if (r_in.n_sets + s_in.n_sets >= 0xffffffffull || r_in.n_tokens + s_in.n_tokens >= 0xffffffffull)
        fail(FGSS_ERR_UNSUPPORTED, "R-S join: more than 2^32-1 records or tokens in total");
    RsInput u;
    const fgss_sets_view r = rs_side_on_device(c, r_in, "r");
    const fgss_sets_view s = rs_side_on_device(c, s_in, "s");
    u.nr = r.n_sets;
    u.ns = s.n_sets;
    u.rid = r.id;
    u.sid = s.id;
    const uint64_t n = u.nr + u.ns, T = r.n_tokens + s.n_tokens;
    uint32_t* upos = c.devT<uint32_t>("rs.u.pos", n + 1);
    uint32_t* ulen = c.devT<uint32_t>("rs.u.len", n + 1);
    uint32_t* utok = c.devT<uint32_t>("rs.u.tok", T + 1);
    u.side = c.devT<uint8_t>("rs.u.side", n + 1);
    u.orig = c.devT<uint32_t>("rs.u.orig", n + 1);
    uint32_t* bad = c.devT<uint32_t>("rs.u.bad", 1);
    FGSS_CK(cudaMemsetAsync(bad, 0, 4, c.stream));
    if (r.n_tokens)
        FGSS_CK(cudaMemcpyAsync(utok, r.tokens, r.n_tokens * 4, cudaMemcpyDeviceToDevice, c.stream));
    if (s.n_tokens)
        FGSS_CK(cudaMemcpyAsync(utok + r.n_tokens, s.tokens, s.n_tokens * 4, cudaMemcpyDeviceToDevice, c.stream));
    if (n) {
        uint64_t* key = c.devT<uint64_t>("rs.u.key", n + 1);
        uint32_t* val = c.devT<uint32_t>("rs.u.val", n + 1);
        k_rs_keys<<<grid_for(n, 256, c.num_sms * 16), 256, 0, c.stream>>>(r.len, (uint32_t)u.nr, s.len,
                                                                        (uint32_t)u.ns, key, val);
        FGSS_LAUNCH_CK();
        radix_sort<uint64_t, uint32_t>(c, key, val, n, nullptr, 0, 48, "rs.u.sort");
        k_rs_union<<<grid_for(n, 256, c.num_sms * 16), 256, 0, c.stream>>>(
            key, (uint32_t)n, r.pos, r.len, r.n_tokens, s.pos, s.len, s.n_tokens, upos, ulen, u.side, u.orig, bad);
        FGSS_LAUNCH_CK();
        uint32_t* h = c.pinnedT<uint32_t>("rs.h.bad", 1);
        FGSS_CK(cudaMemcpyAsync(h, bad, 4, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        if (h[0]) fail(FGSS_ERR_FORMAT, "R-S join: a record's pos + len exceeds its side's n_tokens");
    }
    u.view.id = nullptr;
    u.view.pos = upos;
    u.view.len = ulen;
    u.view.tokens = utok;
    u.view.n_sets = n;
    u.view.n_tokens = T;
    u.view.n_terms = std::max(r.n_terms, s.n_terms);
    u.view.on_device = 1;
    return u;
}

void rs_output(Ctx& c, JoinState& J, const RsInput& u) {
    const uint64_t n = J.n_res;
    uint32_t* q = c.devT<uint32_t>("rs.o.q", n + 1);
    uint32_t* s = c.devT<uint32_t>("rs.o.s", n + 1);
    uint32_t* idq = c.devT<uint32_t>("rs.o.idq", n + 1);
    uint32_t* ids = c.devT<uint32_t>("rs.o.ids", n + 1);
    uint32_t* o = c.devT<uint32_t>("rs.o.o", n + 1);
    float* sim = c.devT<float>("rs.o.sim", n + 1);
    if (n) {
        uint64_t* key = c.devT<uint64_t>("rs.o.key", n + 1);
        uint32_t* val = c.devT<uint32_t>("rs.o.val", n + 1);
        k_rs_remap<<<grid_for(n, 256, c.num_sms * 16), 256, 0, c.stream>>>(J.oq, J.os, n, u.side, u.orig, key, val);
        FGSS_LAUNCH_CK();
        radix_sort<uint64_t, uint32_t>(c, key, val, n, nullptr, 0, bits_needed(u.ns), "rs.o.sort.lo");
        radix_sort<uint64_t, uint32_t>(c, key, val, n, nullptr, 32, 32 + bits_needed(u.nr), "rs.o.sort.hi");
        k_rs_out<<<grid_for(n, 256, c.num_sms * 16), 256, 0, c.stream>>>(key, val, n, u.rid, u.sid, J.oo, J.osim, q, s,
                                                                        idq, ids, o, sim);
        FGSS_LAUNCH_CK();
    }
    J.oq = q;
    J.os = s;
    J.oidq = idq;
    J.oids = ids;
    J.oo = o;
    J.osim = sim;
}

}  // namespace fgss
