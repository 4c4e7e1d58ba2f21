// tokenize.cu -- text -> token sets on the GPU.
//
// Semantics follow the reference's preprocessing and its shipped fixture:
//   lines            src/io.cpp:8-26 (split on '\n', empty lines skipped)
//   lower-case       src/preprocess/string/data.cpp:36-40 (ASCII A-Z only)
//   q-grams          src/preprocess/string/qgram.cpp:20-49 (unpadded; every
//                    repeat becomes its own token "gram"+occurrence); padding
//                    and distinct-gram modes are options
//   term ids         src/preprocess_cli.cpp:266-340: ascending document
//                    frequency; ties by first occurrence (line, position) as
//                    test/data/string/small.txt.3gram.bin shows
//   record layout    ids ascending per record, records by ascending size
//                    (ties by line) in a .bin, i.e. the reverse in memory
// Keys are exact: q <= 8 bytes are packed into 64 bits (the reference hashes
// the gram string with sdbm, src/util.cpp:146-157, which can collide); longer
// grams use a 64-bit FNV-1a hash.  k-mer mode packs canonical k-mers (k <= 32)
// of A/C/G/T into 2k bits, skipping windows with any other byte.
//
// Pipeline: newline compaction -> per-line gram counts -> gram keys ->
// stable radix sorts by gram then line (occurrence numbering / dedup) ->
// stable sort by key' (runs = terms; df = run length; first element = first
// occurrence) -> sort of runs by (df, first occurrence) = term id -> sort of
// (line, id) -> records sorted by (size, line) -> gather in memory order.
#include <string.h>

#include <vector>

#include "ctx.h"
#include "prims.cuh"
#include "tokenize.h"

namespace fgss {

namespace {

__device__ __forceinline__ unsigned char lower_ascii(unsigned char c) {
    return (c <= 'Z' && c >= 'A') ? (unsigned char)(c - ('Z' - 'z')) : c;
}

__global__ void k_flag_newlines(const unsigned char* __restrict__ text, uint64_t n, uint32_t* __restrict__ flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = text[i] == '\n';
}

// Line k spans [start, end); line starts are 0 and every newline + 1.
__global__ void k_lines(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ scan, uint64_t n,
                        uint32_t n_lines, uint64_t* __restrict__ nl_pos) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i]) nl_pos[scan[i]] = i;
    (void)n_lines;
}

// Per raw line: bounds, non-empty flag.
__global__ void k_line_bounds(const uint64_t* __restrict__ nl_pos, uint32_t n_nl, uint64_t n_bytes,
                              uint64_t* __restrict__ lstart, uint32_t* __restrict__ llen,
                              uint32_t* __restrict__ nonempty) {
    const uint32_t nl = n_nl + 1;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nl; k += gridDim.x * blockDim.x) {
        uint64_t s = k == 0 ? 0 : nl_pos[k - 1] + 1;
        uint64_t e = k < n_nl ? nl_pos[k] : n_bytes;
        lstart[k] = s;
        llen[k] = (uint32_t)(e - s);
        nonempty[k] = e > s ? 1u : 0u;
    }
}

__global__ void k_compact_lines(const uint64_t* __restrict__ lstart, const uint32_t* __restrict__ llen,
                                const uint32_t* __restrict__ nonempty, const uint32_t* __restrict__ off, uint32_t nl,
                                uint64_t* __restrict__ ostart, uint32_t* __restrict__ olen) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nl; k += gridDim.x * blockDim.x)
        if (nonempty[k]) {
            ostart[off[k]] = lstart[k];
            olen[off[k]] = llen[k];
        }
}

__device__ __forceinline__ int base2(unsigned char c) {
    switch (lower_ascii(c)) {
        case 'a': return 0;
        case 'c': return 1;
        case 'g': return 2;
        case 't': return 3;
        default: return -1;
    }
}

// Grams per (non-empty) line.
__global__ void k_gram_count(const unsigned char* __restrict__ text, const uint64_t* __restrict__ ls,
                             const uint32_t* __restrict__ ll, uint32_t nlines, TokParams p, uint32_t* __restrict__ g) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; l < nlines; l += warps) {
        int64_t len = ll[l];
        if (p.mode == 0) {
            int64_t c = p.pad ? len + p.q - 1 : len - p.q + 1;
            if (lane_id() == 0) g[l] = c > 0 ? (uint32_t)c : 0u;
            continue;
        }
        // k-mers: windows of k bytes that are all A/C/G/T
        const unsigned char* t = text + ls[l];
        uint32_t cnt = 0;
        for (int64_t s = lane_id(); s + p.q <= len; s += 32) {
            bool ok = true;
            for (int i = 0; i < p.q && ok; i++) ok = base2(t[s + i]) >= 0;
            cnt += ok;
        }
        cnt = warp_sum(cnt);
        if (lane_id() == 0) g[l] = cnt;
    }
}

__device__ __forceinline__ unsigned char padded_at(const unsigned char* t, int64_t len, int64_t i, const TokParams& p) {
    // i indexes the padded line: [pad x (q-1)] line [pad x (q-1)]
    int64_t np = p.pad ? p.q - 1 : 0;
    int64_t j = i - np;
    if (j < 0 || j >= len) return (unsigned char)p.pad_char;
    unsigned char c = t[j];
    return p.lower ? lower_ascii(c) : c;
}

// Gram keys (line-major, position order) and their (line, position) tags.
__global__ void k_gram_fill(const unsigned char* __restrict__ text, const uint64_t* __restrict__ ls,
                            const uint32_t* __restrict__ ll, uint32_t nlines, TokParams p,
                            const uint32_t* __restrict__ goff, uint64_t* __restrict__ key, uint64_t* __restrict__ tag) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; l < nlines; l += warps) {
        int64_t len = ll[l];
        const unsigned char* t = text + ls[l];
        uint32_t o = goff[l];
        if (p.mode == 0) {
            int64_t g = p.pad ? len + p.q - 1 : len - p.q + 1;
            for (int64_t s = lane_id(); s < g; s += 32) {
                uint64_t k;
                if (p.q <= 8) {
                    k = 0;
                    for (int i = 0; i < p.q; i++) k = (k << 8) | padded_at(t, len, s + i, p);
                } else {
                    k = 1469598103934665603ULL;
                    for (int i = 0; i < p.q; i++) {
                        k ^= padded_at(t, len, s + i, p);
                        k *= 1099511628211ULL;
                    }
                }
                key[o + s] = k;
                tag[o + s] = ((uint64_t)l << 32) | (uint32_t)s;
            }
        } else {
            // k-mers: windows are written in position order with a warp-wide compaction
            uint32_t base = o;
            for (int64_t s0 = 0; s0 + p.q <= len; s0 += 32) {
                int64_t s = s0 + lane_id();
                bool ok = s + p.q <= len;
                uint64_t f = 0, r = 0;
                for (int i = 0; i < p.q && ok; i++) {
                    int c = base2(t[s + i]);
                    if (c < 0) { ok = false; break; }
                    f = (f << 2) | (uint64_t)c;
                    r |= (uint64_t)(3 - c) << (2 * i);
                }
                uint32_t m = __ballot_sync(kFull, ok);
                if (ok) {
                    uint32_t d = base + __popc(m & lanemask_lt());
                    key[d] = f < r ? f : r;
                    tag[d] = ((uint64_t)l << 32) | (uint32_t)s;
                }
                base += __popc(m);
            }
        }
    }
}

// After sorting by (line, gram, position): occurrence number (suffix mode) or
// first-of-run flag (distinct mode).  In suffix mode the key becomes
// gram << 16 | occurrence (q <= 6 keeps it within 64 bits).
__global__ void k_occurrence(const uint64_t* __restrict__ key, const uint64_t* __restrict__ tag, uint64_t n,
                             int suffix, uint64_t* __restrict__ key2, uint32_t* __restrict__ keep) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = key[i];
        uint32_t line = (uint32_t)(tag[i] >> 32);
        uint64_t j = i;
        while (j > 0 && key[j - 1] == k && (uint32_t)(tag[j - 1] >> 32) == line) j--;
        uint64_t occ = i - j;
        if (suffix) {
            key2[i] = (k << 16) | (occ < 0xffffu ? occ : 0xffffu);
            keep[i] = 1;
        } else {
            key2[i] = k;
            keep[i] = occ == 0;
        }
    }
}

__global__ void k_compact_tok(const uint64_t* __restrict__ key, const uint64_t* __restrict__ tag,
                              const uint32_t* __restrict__ keep, const uint32_t* __restrict__ off, uint64_t n,
                              uint64_t* __restrict__ okey, uint64_t* __restrict__ otag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (keep[i]) {
            okey[off[i]] = key[i];
            otag[off[i]] = tag[i];
        }
}

// tag (line << 32 | pos) -> global gram index (monotone in (line, pos)) for the first-occurrence order
__global__ void k_tag_index(const uint64_t* __restrict__ tag, const uint32_t* __restrict__ goff, uint64_t n,
                            uint32_t* __restrict__ gidx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t t = tag[i];
        gidx[i] = goff[t >> 32] + (uint32_t)t;
    }
}

// Runs of equal key (sorted): run-start flags
__global__ void k_run_flags(const uint64_t* __restrict__ key, uint64_t n, uint32_t* __restrict__ flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// Run id of every element (exclusive scan of the run-start flags) and the
// start index of every run.
__global__ void k_run_start(const uint32_t* __restrict__ flag, uint32_t* __restrict__ rid, uint64_t n,
                            uint32_t* __restrict__ rstart) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t r = rid[i] + flag[i] - 1;
        rid[i] = r;
        if (flag[i]) rstart[r] = (uint32_t)i;
    }
}

__global__ void k_run_keys2(const uint32_t* __restrict__ rstart, const uint32_t* __restrict__ gidx, uint64_t n,
                            uint32_t nruns, uint64_t* __restrict__ rkey, uint32_t* __restrict__ rval) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += gridDim.x * blockDim.x) {
        uint32_t s = rstart[r];
        uint32_t e = r + 1 < nruns ? rstart[r + 1] : (uint32_t)n;
        uint64_t df = e - s;
        rkey[r] = (df << 32) | gidx[s];  // sorted input: first element of a run is its first occurrence
        rval[r] = r;
    }
}

// rank of every run after the (df, first) sort -> term id per run
__global__ void k_run_ids(const uint32_t* __restrict__ rval_sorted, uint32_t nruns, uint32_t* __restrict__ id_of_run) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nruns; k += gridDim.x * blockDim.x)
        id_of_run[rval_sorted[k]] = k;
}

// tokens -> (line << 32 | id) keys with the position as value
__global__ void k_line_id_keys(const uint32_t* __restrict__ rid, const uint32_t* __restrict__ id_of_run,
                               const uint64_t* __restrict__ tag, uint64_t n, uint64_t* __restrict__ k2,
                               uint32_t* __restrict__ pos) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t t = tag[i];
        k2[i] = (t & 0xffffffff00000000ull) | id_of_run[rid[i]];
        pos[i] = (uint32_t)t;
    }
}

// tokens per line (sorted by line): sizes via run boundaries
__global__ void k_line_bounds2(const uint64_t* __restrict__ k2, uint64_t n, uint32_t* __restrict__ lend,
                               uint32_t* __restrict__ loff) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t l = (uint32_t)(k2[i] >> 32);
        if (i == 0 || (uint32_t)(k2[i - 1] >> 32) != l) loff[l] = (uint32_t)i;
        if (i + 1 == n || (uint32_t)(k2[i + 1] >> 32) != l) lend[l] = (uint32_t)(i + 1);
    }
}

__global__ void k_line_sizes(const uint32_t* __restrict__ lend, const uint32_t* __restrict__ loff, uint32_t nlines,
                             uint32_t* __restrict__ lsz) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nlines; l += gridDim.x * blockDim.x)
        lsz[l] = lend[l] - loff[l];  // both zero for a line without tokens
}

// record sort keys: lines with tokens, key = (size << 32 | line); value = line
__global__ void k_rec_keys(const uint32_t* __restrict__ lsz, uint32_t nlines, uint64_t* __restrict__ rk,
                           uint32_t* __restrict__ rv) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nlines; l += gridDim.x * blockDim.x) {
        rk[l] = ((uint64_t)lsz[l] << 32) | l;
        rv[l] = l;
    }
}

// memory order i = file order reversed; file order = ascending (size, line)
// (empty records sort first in file order and are cut off at the end)
__global__ void k_rec_out(const uint32_t* __restrict__ rv_sorted, const uint32_t* __restrict__ lsz, uint32_t nlines,
                          uint32_t nempty, uint32_t* __restrict__ mline, uint32_t* __restrict__ mid,
                          uint32_t* __restrict__ mlen) {
    const uint32_t nrec = nlines - nempty;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nrec; i += gridDim.x * blockDim.x) {
        uint32_t l = rv_sorted[nlines - 1 - i];
        mline[i] = l;
        mid[i] = l + 1;  // 1-based line number among the non-empty lines
        mlen[i] = lsz[l];
    }
}

__global__ void k_gather_rec(const uint32_t* __restrict__ mline, const uint32_t* __restrict__ moff, uint32_t nrec,
                             const uint32_t* __restrict__ loff, const uint32_t* __restrict__ lsz,
                             const uint64_t* __restrict__ k2, const uint32_t* __restrict__ pos,
                             uint32_t* __restrict__ otok, uint32_t* __restrict__ oloc) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nrec; i += warps) {
        uint32_t l = mline[i], src = loff[l], n = lsz[l], dst = moff[i];
        for (uint32_t j = lane_id(); j < n; j += 32) {
            otok[dst + j] = (uint32_t)k2[src + j];
            oloc[dst + j] = pos[src + j];
        }
    }
}

__global__ void k_count_zero(const uint32_t* __restrict__ lsz, uint32_t n, uint32_t* out) {
    uint32_t c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += lsz[i] == 0;
    c = warp_sum(c);
    if (lane_id() == 0 && c) atomicAdd(out, c);
}

int key_bits(const TokParams& p) {
    if (p.mode == 1) return 2 * p.q;
    if (p.q <= 8) return 8 * p.q;
    return 64;
}

int bits_for32(uint64_t v) {
    int b = 1;
    while (b < 64 && (1ull << b) < v) b++;
    return b;
}

uint32_t read_u32(Ctx& c, const uint32_t* d) {
    uint32_t* h = c.pinnedT<uint32_t>("tk.h", 4);
    FGSS_CK(cudaMemcpyAsync(h, d, 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    return *h;
}

}  // namespace

void tokenize_device(Ctx& c, const char* text, uint64_t n_bytes, const TokParams& p, fgss_sets* out) {
    if (p.q < 1 || p.q > 1024) fail(FGSS_ERR_INVALID, "q must be in [1, 1024] (preprocess_cli.cpp:41,86)");
    if (p.mode == 1 && p.q > 32) fail(FGSS_ERR_INVALID, "k-mers need k <= 32");
    if (p.mode == 0 && p.suffix && p.q > 6)
        fail(FGSS_ERR_UNSUPPORTED, "occurrence-suffix mode supports q <= 6 (gram and occurrence share 64 bits)");
    if (n_bytes >= (1ull << 32)) fail(FGSS_ERR_UNSUPPORTED, "text of 4 GiB or more");
    memset(out, 0, sizeof *out);
    const uint64_t nb = n_bytes;
    unsigned char* dtext = c.devT<unsigned char>("tk.text", nb + 16);
    if (nb) FGSS_CK(cudaMemcpyAsync(dtext, text, nb, cudaMemcpyHostToDevice, c.stream));
    // 1. lines
    uint32_t* flag = c.devT<uint32_t>("tk.flag", nb + 1);
    uint32_t* scan = c.devT<uint32_t>("tk.scan", nb + 1);
    uint32_t* tot = c.devT<uint32_t>("tk.tot", 8);
    FGSS_CK(cudaMemsetAsync(tot, 0, 32, c.stream));
    uint32_t n_nl = 0;
    if (nb) {
        k_flag_newlines<<<grid_for(nb, 256, c.num_sms * 32), 256, 0, c.stream>>>(dtext, nb, flag);
        FGSS_LAUNCH_CK();
        exclusive_scan<uint32_t>(c, flag, scan, nb, nullptr, tot, "tk.s1");
        n_nl = read_u32(c, tot);
    }
    uint64_t* nl_pos = c.devT<uint64_t>("tk.nlpos", (uint64_t)n_nl + 1);
    if (n_nl) {
        k_lines<<<grid_for(nb, 256, c.num_sms * 32), 256, 0, c.stream>>>(flag, scan, nb, n_nl, nl_pos);
        FGSS_LAUNCH_CK();
    }
    const uint32_t nraw = n_nl + 1;
    uint64_t* lstart = c.devT<uint64_t>("tk.lstart", nraw);
    uint32_t* llen = c.devT<uint32_t>("tk.llen", nraw);
    uint32_t* nonempty = c.devT<uint32_t>("tk.ne", nraw);
    uint32_t* noff = c.devT<uint32_t>("tk.noff", nraw);
    k_line_bounds<<<grid_for(nraw, 256), 256, 0, c.stream>>>(nl_pos, n_nl, nb, lstart, llen, nonempty);
    FGSS_LAUNCH_CK();
    exclusive_scan<uint32_t>(c, nonempty, noff, nraw, nullptr, tot + 1, "tk.s2");
    const uint32_t nlines = read_u32(c, tot + 1);
    if (nlines == 0) return;
    uint64_t* ls = c.devT<uint64_t>("tk.ls", nlines);
    uint32_t* ll = c.devT<uint32_t>("tk.ll", nlines);
    k_compact_lines<<<grid_for(nraw, 256), 256, 0, c.stream>>>(lstart, llen, nonempty, noff, nraw, ls, ll);
    FGSS_LAUNCH_CK();
    // 2. grams
    uint32_t* gcnt = c.devT<uint32_t>("tk.gcnt", nlines + 1);
    uint32_t* goff = c.devT<uint32_t>("tk.goff", nlines + 1);
    k_gram_count<<<grid_for((uint64_t)nlines * 32, 256, c.num_sms * 32), 256, 0, c.stream>>>(dtext, ls, ll, nlines, p,
                                                                                            gcnt);
    FGSS_LAUNCH_CK();
    exclusive_scan<uint32_t>(c, gcnt, goff, nlines, nullptr, tot + 2, "tk.s3");
    const uint64_t G = read_u32(c, tot + 2);
    if (G == 0) return;
    uint64_t* key = c.devT<uint64_t>("tk.key", G);
    uint64_t* tag = c.devT<uint64_t>("tk.tag", G);
    k_gram_fill<<<grid_for((uint64_t)nlines * 32, 256, c.num_sms * 32), 256, 0, c.stream>>>(dtext, ls, ll, nlines, p,
                                                                                           goff, key, tag);
    FGSS_LAUNCH_CK();
    const int kb = key_bits(p);
    const int lb = bits_for32(nlines);
    // 3. (line, gram, position) order: stable by gram, then by line
    radix_sort<uint64_t, uint64_t>(c, key, tag, G, nullptr, 0, kb, "tk.sortA");
    {
        // sort by line: the line sits in tag's high half; sort (tag, key) by bits [32, 32+lb)
        radix_sort<uint64_t, uint64_t>(c, tag, key, G, nullptr, 32, 32 + lb, "tk.sortB");
    }
    const bool suffix = p.mode == 0 && p.suffix;
    uint64_t* key2 = c.devT<uint64_t>("tk.key2", G);
    uint32_t* keep = c.devT<uint32_t>("tk.keep", G + 1);
    k_occurrence<<<grid_for(G, 256, c.num_sms * 32), 256, 0, c.stream>>>(key, tag, G, suffix ? 1 : 0, key2, keep);
    FGSS_LAUNCH_CK();
    uint64_t Tn = G;
    uint64_t* tkey = key2;
    uint64_t* ttag = tag;
    if (!suffix) {
        uint32_t* koff = c.devT<uint32_t>("tk.koff", G + 1);
        exclusive_scan<uint32_t>(c, keep, koff, G, nullptr, tot + 3, "tk.s4");
        Tn = read_u32(c, tot + 3);
        tkey = c.devT<uint64_t>("tk.ckey", Tn + 1);
        ttag = c.devT<uint64_t>("tk.ctag", Tn + 1);
        k_compact_tok<<<grid_for(G, 256, c.num_sms * 32), 256, 0, c.stream>>>(key2, tag, keep, koff, G, tkey, ttag);
        FGSS_LAUNCH_CK();
    }
    // 4. terms: stable sort by key' keeps (line, position) order inside a run
    const int kb2 = suffix ? kb + 16 : kb;
    radix_sort<uint64_t, uint64_t>(c, tkey, ttag, Tn, nullptr, 0, kb2 > 64 ? 64 : kb2, "tk.sortC");
    uint32_t* gidx = c.devT<uint32_t>("tk.gidx", Tn + 1);
    k_tag_index<<<grid_for(Tn, 256, c.num_sms * 32), 256, 0, c.stream>>>(ttag, goff, Tn, gidx);
    FGSS_LAUNCH_CK();
    uint32_t* rflag = c.devT<uint32_t>("tk.rflag", Tn + 1);
    uint32_t* rid = c.devT<uint32_t>("tk.rid", Tn + 1);
    k_run_flags<<<grid_for(Tn, 256, c.num_sms * 32), 256, 0, c.stream>>>(tkey, Tn, rflag);
    FGSS_LAUNCH_CK();
    exclusive_scan<uint32_t>(c, rflag, rid, Tn, nullptr, tot + 4, "tk.s5");
    const uint32_t V = read_u32(c, tot + 4);
    uint32_t* rstart = c.devT<uint32_t>("tk.rstart", (uint64_t)V + 1);
    k_run_start<<<grid_for(Tn, 256, c.num_sms * 32), 256, 0, c.stream>>>(rflag, rid, Tn, rstart);
    FGSS_LAUNCH_CK();
    uint64_t* rkey = c.devT<uint64_t>("tk.rkey", (uint64_t)V + 1);
    uint32_t* rval = c.devT<uint32_t>("tk.rval", (uint64_t)V + 1);
    k_run_keys2<<<grid_for(V, 256, c.num_sms * 32), 256, 0, c.stream>>>(rstart, gidx, Tn, V, rkey, rval);
    FGSS_LAUNCH_CK();
    radix_sort<uint64_t, uint32_t>(c, rkey, rval, V, nullptr, 0, 32 + bits_for32((uint64_t)nlines + 1), "tk.sortD");
    uint32_t* id_of_run = c.devT<uint32_t>("tk.idrun", (uint64_t)V + 1);
    k_run_ids<<<grid_for(V, 256, c.num_sms * 32), 256, 0, c.stream>>>(rval, V, id_of_run);
    FGSS_LAUNCH_CK();
    // 5. (line, id) order
    uint64_t* k2 = c.devT<uint64_t>("tk.k2", Tn + 1);
    uint32_t* pos = c.devT<uint32_t>("tk.pos", Tn + 1);
    k_line_id_keys<<<grid_for(Tn, 256, c.num_sms * 32), 256, 0, c.stream>>>(rid, id_of_run, ttag, Tn, k2, pos);
    FGSS_LAUNCH_CK();
    radix_sort<uint64_t, uint32_t>(c, k2, pos, Tn, nullptr, 0, bits_for32((uint64_t)V + 1), "tk.sortE");
    radix_sort<uint64_t, uint32_t>(c, k2, pos, Tn, nullptr, 32, 32 + lb, "tk.sortF");
    // 6. per-line sizes, records by (size, line)
    uint32_t* lsz = c.devT<uint32_t>("tk.lsz", nlines + 1);
    uint32_t* loff = c.devT<uint32_t>("tk.loff", nlines + 1);
    uint32_t* lend = c.devT<uint32_t>("tk.lend", nlines + 1);
    FGSS_CK(cudaMemsetAsync(loff, 0, (uint64_t)nlines * 4, c.stream));
    FGSS_CK(cudaMemsetAsync(lend, 0, (uint64_t)nlines * 4, c.stream));
    k_line_bounds2<<<grid_for(Tn, 256, c.num_sms * 32), 256, 0, c.stream>>>(k2, Tn, lend, loff);
    FGSS_LAUNCH_CK();
    k_line_sizes<<<grid_for(nlines, 256, c.num_sms * 8), 256, 0, c.stream>>>(lend, loff, nlines, lsz);
    FGSS_LAUNCH_CK();
    k_count_zero<<<grid_for(nlines, 256, c.num_sms * 8), 256, 0, c.stream>>>(lsz, nlines, tot + 5);
    FGSS_LAUNCH_CK();
    uint64_t* rk = c.devT<uint64_t>("tk.rk", nlines + 1);
    uint32_t* rv = c.devT<uint32_t>("tk.rv", nlines + 1);
    k_rec_keys<<<grid_for(nlines, 256), 256, 0, c.stream>>>(lsz, nlines, rk, rv);
    FGSS_LAUNCH_CK();
    radix_sort<uint64_t, uint32_t>(c, rk, rv, nlines, nullptr, 0, lb, "tk.sortG");
    radix_sort<uint64_t, uint32_t>(c, rk, rv, nlines, nullptr, 32, 64, "tk.sortH");
    const uint32_t nempty = read_u32(c, tot + 5);
    const uint32_t nrec = nlines - nempty;
    uint32_t* mline = c.devT<uint32_t>("tk.mline", nrec + 1);
    uint32_t* mid = c.devT<uint32_t>("tk.mid", nrec + 1);
    uint32_t* mlen = c.devT<uint32_t>("tk.mlen", nrec + 1);
    uint32_t* moff = c.devT<uint32_t>("tk.moff", nrec + 1);
    if (nrec) {
        k_rec_out<<<grid_for(nrec, 256), 256, 0, c.stream>>>(rv, lsz, nlines, nempty, mline, mid, mlen);
        FGSS_LAUNCH_CK();
        exclusive_scan<uint32_t>(c, mlen, moff, nrec, nullptr, tot + 6, "tk.s6");
    }
    uint32_t* otok = c.devT<uint32_t>("tk.otok", Tn + 1);
    uint32_t* oloc = c.devT<uint32_t>("tk.oloc", Tn + 1);
    if (nrec) {
        k_gather_rec<<<grid_for((uint64_t)nrec * 32, 256, c.num_sms * 32), 256, 0, c.stream>>>(
            mline, moff, nrec, loff, lsz, k2, pos, otok, oloc);
        FGSS_LAUNCH_CK();
    }
    // 7. copy out (host arrays owned by the caller's fgss_sets)
    out->n_sets = nrec;
    out->n_tokens = Tn;
    out->n_terms = V;
    out->id = (uint32_t*)malloc(((uint64_t)nrec + 1) * 4);
    out->len = (uint32_t*)malloc(((uint64_t)nrec + 1) * 4);
    out->pos = (uint32_t*)malloc(((uint64_t)nrec + 1) * 4);
    out->tokens = (uint32_t*)malloc((Tn + 1) * 4);
    out->loc = (uint32_t*)malloc((Tn + 1) * 4);
    if (!out->id || !out->len || !out->pos || !out->tokens || !out->loc) fail(FGSS_ERR_NOMEM, "host allocation");
    if (nrec) {
        FGSS_CK(cudaMemcpyAsync(out->id, mid, (uint64_t)nrec * 4, cudaMemcpyDeviceToHost, c.stream));
        FGSS_CK(cudaMemcpyAsync(out->len, mlen, (uint64_t)nrec * 4, cudaMemcpyDeviceToHost, c.stream));
        FGSS_CK(cudaMemcpyAsync(out->pos, moff, (uint64_t)nrec * 4, cudaMemcpyDeviceToHost, c.stream));
    }
    FGSS_CK(cudaMemcpyAsync(out->tokens, otok, Tn * 4, cudaMemcpyDeviceToHost, c.stream));
    FGSS_CK(cudaMemcpyAsync(out->loc, oloc, Tn * 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    uint32_t mx = 0;
    for (uint32_t i = 0; i < nrec; i++) mx = out->len[i] > mx ? out->len[i] : mx;
    out->max_len = mx;
}

}  // namespace fgss
